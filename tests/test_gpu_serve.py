"""The serving loop: continuous batching of mixed requests.  Each result is
the same alone and in the mix, and equals the oracle; admission respects the
memory budget; failures stay per request."""
import random
import threading

import numpy as np
import pytest

import cellato_b200 as cb
from oracle import oracle as O

pytestmark = pytest.mark.gpu

PROBS = {0: [0.5, 0.5], 1: [0.6, 0.05, 0.05, 0.3], 2: [0.125] * 8}


def specs(n, seed):
    rng = random.Random(seed)
    return [(rng.randrange(3), 32 * rng.randint(1, 24), rng.randint(1, 70), rng.choice([0, 1, 2, 7, 20, 65, 130]),
             rng.randrange(1 << 30)) for _ in range(n)]


def oracle_checksum(a, x, y, steps, seed):
    cells = O.init_cells(x, y, seed, O.thresholds(PROBS[a]))
    return O.checksum(O.run_standard(a, cells, steps))


def test_each_result_is_the_same_alone_and_in_the_mix(cuda):
    mix = specs(30, 1)
    with cb.Server(chunk_steps=16) as srv:
        ids = [srv.submit(a, x, y, s, seed, PROBS[a]) for (a, x, y, s, seed) in mix]
        srv.drain(120)
        in_mix = [srv.wait(i)["checksum"] for i in ids]
    for (a, x, y, s, seed), ck in zip(mix, in_mix):
        assert ck == oracle_checksum(a, x, y, s, seed), (a, x, y, s)
    with cb.Server(chunk_steps=16) as srv:  # alone: one request per server round
        for (a, x, y, s, seed), ck in zip(mix[:8], in_mix[:8]):
            rid = srv.submit(a, x, y, s, seed, PROBS[a])
            assert srv.wait(rid, 60)["checksum"] == ck


def test_host_cells_in_and_out(cuda):
    with cb.Server(chunk_steps=8) as srv:
        jobs = []
        for i, (a, x, y, s, seed) in enumerate(specs(10, 2)):
            cells = O.init_cells(x, y, seed, O.thresholds(PROBS[a]))
            jobs.append((a, cells, s, srv.submit(a, x, y, s, cells=cells, want_cells=True)))
        srv.drain(120)
        for a, cells, s, rid in jobs:
            assert srv.wait(rid)["state"] == "done"
            assert (srv.result_cells(rid) == O.run_standard(a, cells, s)).all()
        bad = np.zeros((4, 32), dtype=np.uint8)
        bad[1, 1] = 3  # not a game-of-life state
        rid = srv.submit(0, 32, 4, 5, cells=bad)
        with pytest.raises(cb.StateError):
            srv.wait(rid, 30)


def test_per_request_path_gives_the_same_results(cuda):
    mix = specs(12, 3)
    out = []
    for per_request in (False, True):
        with cb.Server(per_request=per_request) as srv:
            ids = [srv.submit(a, x, y, s, seed, PROBS[a]) for (a, x, y, s, seed) in mix]
            srv.drain(120)
            out.append([srv.status(i)["checksum"] for i in ids])
    assert out[0] == out[1]


def test_admission_respects_the_memory_budget(cuda):
    # each request holds 2 x 1 plane x 256x256/8 = 16 KiB; the budget fits 3
    budget = 3 * 16384 + 100
    with cb.Server(memory_budget=budget, chunk_steps=4) as srv:
        ids = [srv.submit(0, 256, 256, 40, seed=i, probs=PROBS[0]) for i in range(12)]
        srv.drain(120)
        st = [srv.status(i) for i in ids]
        with pytest.raises(MemoryError, match="budget"):
            srv.submit(0, 1024, 1024, 1, seed=1)
    events = sorted([(s["admit_s"], 1) for s in st] + [(s["done_s"], -1) for s in st], key=lambda e: (e[0], e[1]))
    live = peak = 0
    for _, d in events:
        live += d
        peak = max(peak, live)
    assert peak <= 3
    for (i, s) in zip(range(12), st):
        assert s["checksum"] == oracle_checksum(0, 256, 256, 40, i)


def test_injected_allocation_failure_fails_only_that_request(cuda):
    mix = specs(6, 4)
    with cb.Server(fail_alloc_at=3) as srv:
        ids = [srv.submit(a, x, y, s, seed, PROBS[a]) for (a, x, y, s, seed) in mix]
        srv.drain(60)
        states = [srv.status(i)["state"] for i in ids]
        assert states.count("failed") == 1 and states[2] == "failed"
        with pytest.raises(MemoryError, match="injected"):
            srv.wait(ids[2])
        for (a, x, y, s, seed), rid in zip(mix, ids):
            if rid != ids[2]:
                assert srv.status(rid)["checksum"] == oracle_checksum(a, x, y, s, seed)
        stats = srv.stats()
        assert stats["completed"] == 5 and stats["failed"] == 1


def test_concurrent_submitters(cuda):
    mix = specs(40, 5)
    ids = [None] * len(mix)
    with cb.Server(chunk_steps=32) as srv:
        def worker(k):
            for j in range(k, len(mix), 4):
                a, x, y, s, seed = mix[j]
                ids[j] = srv.submit(a, x, y, s, seed, PROBS[a])
        threads = [threading.Thread(target=worker, args=(k,)) for k in range(4)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        srv.drain(120)
        for (a, x, y, s, seed), rid in zip(mix, ids):
            assert srv.status(rid)["checksum"] == oracle_checksum(a, x, y, s, seed)


@pytest.mark.parametrize("direct_cells", [1, 2048, -1])
def test_large_requests_through_the_strip_kernels_match_the_oracle(cuda, direct_cells):
    # direct_cells = 1: every request advances by strip passes on the second stream;
    # 2048: a mix of batch-kernel and strip-pass requests; -1: none of them.
    mix = specs(24, 7)
    with cb.Server(chunk_steps=16, direct_cells=direct_cells) as srv:
        ids = [srv.submit(a, x, y, s, seed, PROBS[a]) for (a, x, y, s, seed) in mix]
        srv.drain(120)
        got = [srv.wait(i)["checksum"] for i in ids]
    for (a, x, y, s, seed), ck in zip(mix, got):
        assert ck == oracle_checksum(a, x, y, s, seed), (a, x, y, s, direct_cells)


def test_large_request_cells_out_through_the_strip_kernels(cuda):
    with cb.Server(chunk_steps=8, direct_cells=1000) as srv:
        jobs = []
        for (a, x, y, s, seed) in specs(8, 9):
            cells = O.init_cells(x, y, seed, O.thresholds(PROBS[a]))
            jobs.append((a, cells, s, srv.submit(a, x, y, s, cells=cells, want_cells=True)))
        srv.drain(120)
        for a, cells, s, rid in jobs:
            assert (srv.result_cells(rid) == O.run_standard(a, cells, s)).all()
