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


def _stream_of(handle):
    import torch
    return torch.cuda.ExternalStream(handle) if handle else torch.cuda.default_stream()


@pytest.mark.parametrize("a,k", [(0, 8), (1, 32), (2, 4)])
def test_band_run_single_rank_with_exchange_stream(cuda, a, k):
    # cb2_band_run with a self-exchange enqueued on a second stream: the
    # interior runs while the copies land, the edges after them.
    torch = cuda
    x, rows, steps = 2048, 200, 45
    b = BandGrid(a, x, rows)
    b.fill_random(5, PROBS[a])
    g, B = b.ghost, b.band
    calls = []

    def exchange(user, buffer, kk, stream):
        p = b.bufs[buffer]
        with torch.cuda.stream(_stream_of(stream)):
            p[:, g - kk:g, :].copy_(p[:, g + B - kk:g + B, :])
            p[:, g + B:g + B + kk, :].copy_(p[:, g:g + kk, :])
        calls.append(kk)
        return 0

    fn = _abi.HALO_EXCHANGE_FN(exchange)
    side = torch.cuda.Stream()
    res = ctypes.c_int()
    _abi.check(_abi.lib.cb2_band_run(a, _planes(b.bufs[0]), _planes(b.bufs[1]), x, B, g, 0, steps, 42, 0, rows,
                                     ctypes.byref(_abi.tuning(k)), fn, None, None, side.cuda_stream,
                                     ctypes.byref(res)))
    torch.cuda.synchronize()
    b.cur = res.value
    from cellato_b200.bands import schedule
    assert calls == schedule(steps, k, g)
    ck, planes = global_run(a, x, rows, steps, 5)
    assert b.checksum() == ck
    assert (b.band_planes_host().numpy() == planes).all()


@pytest.mark.parametrize("a,k", [(0, 16), (2, 8)])
def test_band_run_two_bands_on_one_gpu(cuda, a, k):
    # Two ranks emulated on one GPU through cb2_band_run, one pass per call,
    # rank 0 then rank 1: each exchange copies from the other band's buffer
    # that holds the generation being advanced (rank 0's previous buffer once
    # it has moved on), so nothing waits on another launch.
    torch = cuda
    x, rows, steps = 4096, 192, 40
    bands = [BandGrid(a, x, rows, rank=r, world=2) for r in range(2)]
    for b in bands:
        b.fill_random(9, PROBS[a])
    g, B = bands[0].ghost, bands[0].band
    gen = [0, 0]

    def make_exchange(r):
        def exchange(user, buffer, kk, stream):
            me, other = bands[r], bands[1 - r]
            src = other.bufs[other.cur if gen[1 - r] == gen[r] else 1 - other.cur]
            dst = (me.bufs[me.cur], me.bufs[1 - me.cur])[buffer]  # the (a, b) pair passed below
            with torch.cuda.stream(_stream_of(stream)):
                dst[:, g - kk:g, :].copy_(src[:, g + B - kk:g + B, :])
                dst[:, g + B:g + B + kk, :].copy_(src[:, g:g + kk, :])
            return 0
        return _abi.HALO_EXCHANGE_FN(exchange)

    fns = [make_exchange(r) for r in range(2)]
    side = torch.cuda.Stream()
    for kk in [k] * (steps // k) + ([steps % k] if steps % k else []):
        for r, b in enumerate(bands):
            res = ctypes.c_int()
            bufs = (b.bufs[b.cur], b.bufs[1 - b.cur])
            _abi.check(_abi.lib.cb2_band_run(a, _planes(bufs[0]), _planes(bufs[1]), x, B, g, gen[r], kk, 42,
                                             b.row0, rows, ctypes.byref(_abi.tuning(kk)), fns[r], None, None,
                                             side.cuda_stream, ctypes.byref(res)))
            b.cur = b.cur ^ res.value
            gen[r] += kk
    torch.cuda.synchronize()
    ck, planes = global_run(a, x, rows, steps, 9)
    sums = [sum(v) for v in zip(*[b.local_checksum() for b in bands])]
    assert sums == ck
    got = np.concatenate([b.band_planes_host().numpy() for b in bands], axis=1)
    assert (got == planes).all()


def test_band_run_python_overlap_path(cuda):
    # BandGrid.run's interior/edge split (taken when world > 1) on one GPU,
    # with the NCCL exchange replaced by copies from a second band.
    torch = cuda
    from cellato_b200 import bands as bands_mod
    a, x, rows, steps = 0, 2048, 128, 37
    bands = [BandGrid(a, x, rows, rank=r, world=2) for r in range(2)]
    for b in bands:
        b.fill_random(3, PROBS[a])
    g, B = bands[0].ghost, bands[0].band
    passes = []

    def fake_post(planes, ghost, band_rows, k, rank, world, group=None):
        other = bands[1 - rank]
        src = other.bufs[other.cur if rank == 0 else 1 - other.cur]
        passes.append(k)

        def finish():
            planes[:, ghost - k:ghost, :].copy_(src[:, ghost + band_rows - k:ghost + band_rows, :])
            planes[:, ghost + band_rows:ghost + band_rows + k, :].copy_(src[:, ghost:ghost + k, :])
        return finish

    real = bands_mod.post_halos
    bands_mod.post_halos = fake_post
    try:
        for kk in bands_mod.schedule(steps, 8, g):
            for b in bands:
                b.run(kk, temporal_steps=kk)
    finally:
        bands_mod.post_halos = real
    torch.cuda.synchronize()
    ck, planes = global_run(a, x, rows, steps, 3)
    got = np.concatenate([b.band_planes_host().numpy() for b in bands], axis=1)
    assert (got == planes).all()
    assert passes == [kk for kk in bands_mod.schedule(steps, 8, g) for _ in range(2)]
