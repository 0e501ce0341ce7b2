"""Row bands across ranks, on CPU with gloo (world sizes 2 and 3): the halo
exchange (cellato_b200.bands.post_halos / exchange_halos, the code the GPU
ranks run over NCCL) and the whole band run -- BandGrid.run's pass schedule
(cb2_band_schedule), with the exchange posted before the band interior and
completed before the two edges -- against the oracle on the global grid.
Only the kernel is replaced: each pass is computed by the oracle on the
window of rows it reads (test infrastructure); on GPUs it is cb2_band_pass_at."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _init(rank, world, port):
    import sys
    sys.path.insert(0, ROOT)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)


def _exchange_worker(rank, world, port, ghost, band, k, out):
    _init(rank, world, port)
    from cellato_b200.bands import exchange_halos
    P, words = 2, 3
    t = torch.full((P, band + 2 * ghost, words), -1, dtype=torch.int32)
    for p in range(P):
        for r in range(band):
            t[p, ghost + r, :] = (rank * 1000 + r) * 10 + p
    exchange_halos(t, ghost, band, k, rank, world)
    up, down = (rank - 1) % world, (rank + 1) % world
    ok = True
    for p in range(P):
        for j in range(k):
            ok &= bool((t[p, ghost - k + j] == (up * 1000 + band - k + j) * 10 + p).all())
            ok &= bool((t[p, ghost + band + j] == (down * 1000 + j) * 10 + p).all())
    out[rank] = int(ok)
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_exchange_halos_gloo(world):
    out = mp.Manager().dict()
    mp.spawn(_exchange_worker, args=(world, _free_port(), 4, 6, 3, out), nprocs=world, join=True)
    assert [out[r] for r in range(world)] == [1] * world


def _oracle_band_grid(automaton, x, rows, rank, world, ghost):
    """A BandGrid on CPU tensors whose pass is the oracle instead of the kernel."""
    from cellato_b200.bands import BandGrid
    from oracle import oracle as O

    class OracleBands(BandGrid):
        def _pass(self, src, dst, row_first, rows_out, k, time_step, tuning, stream):
            lo, hi = row_first - k, row_first + rows_out + k  # the rows a pass of k generations reads
            window = src[:, lo:hi, :].contiguous().numpy().view(np.uint8).reshape(-1)
            cells = O.unpack("bit_planes", window, x, hi - lo, self.P, 32)
            nxt = O.run_standard(self.automaton, cells, k)  # rows within k of the window's edges are junk
            new = O.pack("bit_planes", nxt, self.P, 32).view(np.int32).reshape(self.P, hi - lo, x // 32)
            dst[:, row_first:row_first + rows_out] = torch.from_numpy(new[:, k:k + rows_out].copy())

    return OracleBands(automaton, x, rows, rank=rank, world=world, ghost=ghost, device=torch.device("cpu"))


def _bands_worker(rank, world, port, automaton, x, rows, steps, k, ghost, out):
    _init(rank, world, port)
    from oracle import oracle as O
    probs = {0: [0.5, 0.5], 1: [0.6, 0.05, 0.05, 0.3], 2: [0.125] * 8}[automaton]
    P = O.PLANES[automaton]
    cells = O.init_cells(x, rows, 99, O.thresholds(probs))
    b = _oracle_band_grid(automaton, x, rows, rank, world, ghost)
    idx = [(b.row0 - ghost + i) % rows for i in range(b.rows_total)]
    b.planes.copy_(torch.from_numpy(O.pack("bit_planes", cells[idx], P, 32).view(np.int32)
                                    .reshape(P, b.rows_total, x // 32)))
    passes = b.run(steps, temporal_steps=k)
    mine = O.unpack("bit_planes", b.planes[:, ghost:ghost + b.band].contiguous().numpy().view(np.uint8).reshape(-1),
                    x, b.band, P, 32)
    gathered = [torch.zeros_like(torch.from_numpy(mine)) for _ in range(world)]
    dist.all_gather(gathered, torch.from_numpy(mine.copy()))
    if rank == 0:
        full = np.concatenate([g.numpy() for g in gathered], axis=0)
        out["ok"] = bool((full == O.run_standard(automaton, cells, steps)).all())
        out["passes"] = passes
    dist.destroy_process_group()


@pytest.mark.parametrize("world,automaton,k", [(2, 0, 4), (3, 1, 4), (2, 2, 8), (3, 0, 16)])
def test_band_run_matches_global_oracle(world, automaton, k):
    # Bands of 24 rows: k = 4 and 8 take the interior/edge split, k = 16 the
    # whole-band pass after the exchange; 21 steps end with remainder passes.
    out = mp.Manager().dict()
    ghost = max(5, k)
    mp.spawn(_bands_worker, args=(world, _free_port(), automaton, 64, 24 * world, 21, k, ghost, out), nprocs=world,
             join=True)
    assert out["ok"]
    assert out["passes"] == len(_schedule(21, k, ghost))


def _schedule(steps, k, ghost):
    import sys
    sys.path.insert(0, ROOT)
    from cellato_b200.bands import schedule
    return schedule(steps, k, ghost)


def test_band_schedule():
    assert _schedule(45, 32, 32) == [32, 8, 4, 1]
    assert _schedule(64, 32, 16) == [16, 16, 16, 16]
    assert _schedule(0, 8, 32) == []
    assert _schedule(7, 1, 32) == [1] * 7
    from cellato_b200 import _abi
    assert _abi.lib.cb2_band_schedule(5, 0, 32, None, 0) == _abi.CB2_EINVAL


def _checksum_worker(rank, world, port, out):
    _init(rank, world, port)
    from cellato_b200.bands import BandGrid
    b = BandGrid(0, 64, 32 * world, rank=rank, world=world, ghost=4, device=torch.device("cpu"))
    # Sums modulo 2^64 (negative state values wrap, as the reference's
    # uint64 sums do) must survive the int64 all-reduce.
    big = [(1 << 64) - 5 - i if i % 2 else (1 << 63) + i for i in range(16)]
    b.local_checksum = lambda values=None: list(big)
    out[rank] = b.checksum()
    dist.destroy_process_group()


def test_band_checksum_sums_modulo_2_64():
    out = mp.Manager().dict()
    mp.spawn(_checksum_worker, args=(2, _free_port(), out), nprocs=2, join=True)
    want = [(2 * ((1 << 64) - 5 - i if i % 2 else (1 << 63) + i)) % (1 << 64) for i in range(16)]
    assert out[0] == want and out[1] == want
