"""Band kernels on one GPU: a single rank (ghost rows from its own band) and
two bands emulated on one device (halo rows copied between them) reproduce
the single-grid run on the global grid."""
import ctypes

import numpy as np
import pytest

import cellato_b200 as cb
from cellato_b200 import _abi
from cellato_b200.bands import BandGrid, _planes

pytestmark = pytest.mark.gpu

PROBS = {0: [0.65, 0.35], 1: [0.6, 0.05, 0.05, 0.3], 2: [0.125] * 8}


def global_run(a, x, rows, steps, seed):
    with cb.DeviceGrid(a, x, rows) as g:
        g.fill_random(seed, PROBS[a])
        g.run(steps)
        return g.checksum(), g.download("bit_planes", 32).data.view(np.int32).reshape(-1, rows, x // 32)


@pytest.mark.parametrize("a", [0, 1, 2])
def test_single_rank_band_equals_grid(cuda, a):
    x, rows, steps = 2048, 200, 37
    b = BandGrid(a, x, rows)
    b.fill_random(5, PROBS[a])
    b.run(steps)
    ck, planes = global_run(a, x, rows, steps, 5)
    assert b.checksum() == ck
    assert (b.band_planes_host().numpy() == planes).all()


@pytest.mark.parametrize("a,k", [(0, 16), (1, 8), (2, 4), (0, 32), (2, 32)])
def test_two_bands_on_one_gpu_equal_the_global_grid(cuda, a, k):
    torch = cuda
    x, rows, steps = 4096, 96, 45
    bands = [BandGrid(a, x, rows, rank=r, world=2) for r in range(2)]
    for b in bands:
        b.fill_random(9, PROBS[a])
    g, B = bands[0].ghost, bands[0].band
    left = steps
    t = _abi.tuning()
    while left > 0:
        kk = k
        while kk > left:
            kk //= 2
        for r, b in enumerate(bands):  # halo exchange as the ranks would do it
            other = bands[1 - r].planes
            b.planes[:, g - kk:g, :] = other[:, g + B - kk:g + B, :]
            b.planes[:, g + B:g + B + kk, :] = other[:, g:g + kk, :]
        for b in bands:
            _abi.check(_abi.lib.cb2_band_pass(b.automaton, _planes(b.bufs[b.cur]), _planes(b.bufs[1 - b.cur]), x,
                                              b.rows_total, g, B, kk, ctypes.byref(t), None))
            b.cur ^= 1
        left -= kk
    torch.cuda.synchronize()
    ck, planes = global_run(a, x, rows, steps, 9)
    sums = [sum(v) for v in zip(*[b.local_checksum() for b in bands])]
    assert sums == ck
    got = np.concatenate([b.band_planes_host().numpy() for b in bands], axis=1)
    assert (got == planes).all()


def test_band_pass_rejects_too_few_ghost_rows(cuda):
    b = BandGrid(0, 256, 64, ghost=4)
    t = _abi.tuning()
    rc = _abi.lib.cb2_band_pass(0, _planes(b.bufs[0]), _planes(b.bufs[1]), 256, b.rows_total, 4, 64, 8,
                                ctypes.byref(t), None)
    assert rc == _abi.CB2_EINVAL and "ghost rows" in _abi.last_error()
