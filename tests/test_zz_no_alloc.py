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


def _existing(torch, a, img, x, y, steps, tuning):
    """The reference result: cb2_run_bit_planes with two caller-owned buffers."""
    P = O.PLANES[a]
    buf_a = torch.from_numpy(img.view(np.int32).copy()).cuda()
    buf_b = torch.zeros_like(buf_a)
    res = ctypes.c_int()
    _abi.check(_abi.lib.cb2_run_bit_planes(a, _planes(buf_a, P, x, y), _planes(buf_b, P, x, y), x, y, steps,
                                           ctypes.byref(tuning), None, ctypes.byref(res)))
    torch.cuda.synchronize()
    return (buf_b if res.value else buf_a).cpu().numpy().view(np.uint8)


def _in_place(torch, a, img, x, y, steps, tuning):
    P = O.PLANES[a]
    buf = torch.from_numpy(img.view(np.int32).copy()).cuda()
    _abi.check(_abi.lib.cb2_run_bit_planes_in_place(a, _planes(buf, P, x, y), x, y, steps, ctypes.byref(tuning),
                                                    None))
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
        got = _in_place(torch, a, img, x, y, steps, t)
        assert got.tobytes() == want.tobytes(), (a, x, y, steps)
        assert (O.unpack("bit_planes", got, x, y, O.PLANES[a], 32) == O.run_standard(a, cells, steps)).all()


def test_in_place_rejects_grids_beyond_the_scratch(cuda):
    torch = cuda
    x, y = 8192, 8192  # 3 planes x 8 MiB > 16 MiB
    buf = torch.zeros(3 * x * y // 32, dtype=torch.int32, device="cuda")
    rc = _abi.lib.cb2_run_bit_planes_in_place(2, _planes(buf, 3, x, y), x, y, 4, None, None)
    assert rc == _abi.CB2_EINVAL
    assert "exceeds" in _abi.last_error() and str(16 << 20) in _abi.last_error()
