"""GPU parity against the reference's OWN CUDA traversers (simple and temporal,
bit_planes, 64-bit words), compiled from its headers into
oracle/_ref/libcellato_ref_cuda.so: the same seeded planes advanced by both
must give the same cells.  Skipped where that library was not built."""
import os

import numpy as np
import pytest

import cellato_b200 as cb

pytestmark = pytest.mark.gpu

LIB = os.path.join(os.path.dirname(__file__), "..", "oracle", "_ref", "libcellato_ref_cuda.so")
PROBS = {0: [0.5, 0.5], 1: [0.6, 0.05, 0.05, 0.3], 2: [0.125] * 8}


@pytest.fixture(scope="module")
def refcuda(cuda):
    if not os.path.exists(LIB):
        pytest.skip("reference CUDA traversers not built (oracle/_ref/libcellato_ref_cuda.so)")
    from oracle import ref_cuda_bench as R
    return R.load()


def seeded_planes(a, x, y, seed):
    with cb.DeviceGrid(a, x, y) as g:
        g.fill_random(seed, PROBS[a])
        return np.ascontiguousarray(g.download("bit_planes", 64).data)


def our_run(a, x, y, planes, steps, **plan):
    with cb.DeviceGrid(a, x, y) as g:
        g.upload(cb.HostGrid(a, "bit_planes", 64, x, y, planes))
        g.run(steps, **plan)
        return np.ascontiguousarray(g.download("bit_planes", 64).data)


@pytest.mark.parametrize("a", [0, 1, 2])
def test_reference_simple_kernel_equals_ours(refcuda, a):
    from oracle import ref_cuda_bench as R
    x, y = 2048, 520  # 32 words wide, a multiple of the 8-row block
    planes = seeded_planes(a, x, y, 11 + a)
    ref, _ = R.ref_run(refcuda, a, 0, x, y, 0, 37, 0, 0, 8, planes)
    for plan in (dict(), dict(temporal_steps=8, words_per_lane=1), dict(temporal_steps=32, rows_per_step=4)):
        assert np.array_equal(our_run(a, x, y, planes, 37, **plan), ref), plan


@pytest.mark.parametrize("a,k", [(0, 4), (0, 8), (1, 2), (2, 4)])
def test_reference_temporal_kernel_equals_ours(refcuda, a, k):
    from oracle import ref_cuda_bench as R
    x = 3840  # 60 words: two 30-word temporal tiles across
    eff = 32 - 2 * k
    y = eff * (640 // eff)
    planes = seeded_planes(a, x, y, 5 + a)
    steps = 48
    ref, _ = R.ref_run(refcuda, a, 1, x, y, 0, steps, k, 32, 8, planes)
    assert np.array_equal(our_run(a, x, y, planes, steps), ref)
