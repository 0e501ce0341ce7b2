"""cb2_run_bit_planes_in_place: the allocation-free entry point.

Callers that cannot call cudaMalloc (a host application that owns every
device byte through its own pool, or a step loop that must not allocate)
hand over only the grid; the second buffer is the library's static device
scratch.  Through the C-ABI, its result must equal the existing entry point's
(cb2_run_bit_planes with a caller-owned second buffer) bit for bit, on two
calls in a row -- the second call must not see anything the first left in
the shared scratch.  This file sorts last so that a run stopping at the first
failure has run every other test first; it also passes alone in a fresh
process.
"""
import ctypes

import numpy as np
import pytest

import cellato_b200 as cb
from cellato_b200 import _abi
from oracle import oracle as O

pytestmark = pytest.mark.gpu

PROBS = {0: [0.5, 0.5], 1: [0.6, 0.05, 0.05, 0.3], 2: [0.125] * 8}


def _planes(buf, P, x, y):
    plane_bytes = x * y // 8
    return (ctypes.c_void_p * P)(*[buf.data_ptr() + p * plane_bytes for p in range(P)])


def _n_planes(a):
    return cb.automaton_info(a)[1]


def _existing(torch, a, img, x, y, steps, tuning, time_step=0, seed=42):
    """The reference result: cb2_run_bit_planes_at with two caller-owned buffers."""
    P = _n_planes(a)
    buf_a = torch.from_numpy(img.view(np.int32).copy()).cuda()
    buf_b = torch.zeros_like(buf_a)
    res = ctypes.c_int()
    _abi.check(_abi.lib.cb2_run_bit_planes_at(a, _planes(buf_a, P, x, y), _planes(buf_b, P, x, y), x, y, time_step,
                                              steps, seed, ctypes.byref(tuning), None, ctypes.byref(res)))
    torch.cuda.synchronize()
    return (buf_b if res.value else buf_a).cpu().numpy().view(np.uint8)


def _in_place(torch, a, img, x, y, chunks, tuning, seed=42):
    """A step loop of in-place calls, one per entry of `chunks` (generations),
    each starting at the running generation count."""
    P = _n_planes(a)
    buf = torch.from_numpy(img.view(np.int32).copy()).cuda()
    t = 0
    for steps in chunks:
        _abi.check(_abi.lib.cb2_run_bit_planes_in_place(a, _planes(buf, P, x, y), x, y, t, steps, seed,
                                                        ctypes.byref(tuning), None))
        t += steps
    torch.cuda.synchronize()
    return buf.cpu().numpy().view(np.uint8)


def test_in_place_matches_existing_entry_point_twice(cuda):
    torch = cuda
    # Two calls in a row with different automata, sizes and pass parity: the
    # first leaves its last generation in the shared scratch (odd pass count).
    calls = [(0, 1024, 512, 37, _abi.tuning(8)), (1, 2048, 256, 20, _abi.tuning(4)),
             (2, 4096, 160, 13, _abi.tuning(0))]
    for a, x, y, steps, t in calls:
        cells = O.init_cells(x, y, 100 + a, O.thresholds(PROBS[a]))
        img = O.pack("bit_planes", cells, O.PLANES[a], 32)
        want = _existing(torch, a, img, x, y, steps, t)
        got = _in_place(torch, a, img, x, y, [steps], t)
        assert got.tobytes() == want.tobytes(), (a, x, y, steps)
        assert (O.unpack("bit_planes", got, x, y, O.PLANES[a], 32) == O.run_standard(a, cells, steps)).all()


@pytest.mark.parametrize("name", ["critters", "lightning-forest"])
def test_in_place_step_loop_follows_time_and_seed(cuda, name):
    # A Margolus rule (reads the generation's parity) and a stochastic rule
    # (draws keyed by seed and generation): a loop of in-place calls that
    # passes its running generation count must equal one run of the whole
    # span, the existing entry point, and the reference CPU traverser.
    torch = cuda
    if name not in cb.AUTOMATA:
        pytest.fail(f"library built without the lowered DSL automaton {name}")
    a = cb.AUTOMATA[name]
    x, y, seed = 1056, 96, 7
    chunks = [7, 6, 8]
    _, P, states = cb.automaton_info(a)
    probs = {"critters": [0.5, 0.5], "lightning-forest": [0.3, 0.6, 0.1]}[name]
    cells = O.init_cells(x, y, 300, O.thresholds(probs))
    img = O.pack("bit_planes", cells, P, 32)
    t = _abi.tuning(0)
    want = _existing(torch, a, img, x, y, sum(chunks), t, seed=seed)
    for _ in range(2):  # twice in a row through the shared scratch
        got = _in_place(torch, a, img, x, y, chunks, t, seed=seed)
        assert got.tobytes() == want.tobytes(), name
    if O.ref_available():
        ref_cells, _ = O.ref_run_named(name, cells, sum(chunks), seed=seed)
        assert (O.unpack("bit_planes", got, x, y, P, 32) == ref_cells).all(), name


def test_in_place_rejects_grids_beyond_the_scratch(cuda):
    torch = cuda
    x, y = 8192, 8192  # 3 planes x 8 MiB > 16 MiB
    buf = torch.zeros(3 * x * y // 32, dtype=torch.int32, device="cuda")
    rc = _abi.lib.cb2_run_bit_planes_in_place(2, _planes(buf, 3, x, y), x, y, 0, 4, 42, None, None)
    assert rc == _abi.CB2_EINVAL
    assert "exceeds" in _abi.last_error() and str(16 << 20) in _abi.last_error()
