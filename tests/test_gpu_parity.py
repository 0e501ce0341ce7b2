"""GPU parity: the sm_100a strip kernels, the device generator, the layout
conversions and the device checksum, all called through the C-ABI, against
the oracle and the golden fixtures produced by Cellato itself.  Bit-exact."""
import random

import numpy as np
import pytest

import cellato_b200 as cb
from oracle import oracle as O
from tests.golden.make_golden import unpack_cells

pytestmark = pytest.mark.gpu

PROBS = {0: [0.5, 0.5], 1: [0.6, 0.05, 0.05, 0.3], 2: [0.125] * 8}
PLANS = [dict(), dict(temporal_steps=1), dict(temporal_steps=2, words_per_lane=1),
         dict(temporal_steps=4, tile_rows=5), dict(temporal_steps=8, words_per_lane=2, tile_rows=1),
         dict(temporal_steps=8, words_per_lane=1, tile_rows=64), dict(temporal_steps=8, words_per_lane=4),
         dict(temporal_steps=16, words_per_lane=2, levels_per_warp=2),
         dict(temporal_steps=16, words_per_lane=1, levels_per_warp=4, tile_rows=3),
         dict(temporal_steps=8, words_per_lane=2, levels_per_warp=2),
         dict(temporal_steps=32), dict(temporal_steps=32, words_per_lane=2, levels_per_warp=4, rows_per_step=4,
                                       tile_rows=7),
         dict(temporal_steps=16, words_per_lane=2, levels_per_warp=8, rows_per_step=2, tile_rows=1)]


def variants(a):
    """Every instantiated (K, V, L, rows per step) of automaton a."""
    return cb.variants(a)


def device_run(automaton, cells, steps, **plan):
    y, x = cells.shape
    with cb.DeviceGrid(automaton, x, y) as g:
        g.upload_cells(cells)
        g.run(steps, **plan)
        return g.cells(), g.checksum_str()


def test_fill_random_matches_oracle(cuda):
    for a in (0, 1, 2):
        for (x, y, seed) in [(64, 32, 1), (1024, 64, 42), (32, 7, 3), (96, 100, 12345)]:
            thr = cb.thresholds(PROBS[a])
            with cb.DeviceGrid(a, x, y) as g:
                g.fill_random(seed, thr=thr)
                assert (g.cells() == O.init_cells(x, y, seed, thr)).all(), (a, x, y)


@pytest.mark.parametrize("plan", PLANS, ids=lambda p: ",".join(f"{k}={v}" for k, v in p.items()) or "auto")
def test_golden_cases(cuda, golden, plan):
    cases, arrays = golden
    for c in cases:
        a, x, y = c["automaton"], c["x"], c["y"]
        if x * y > 2 ** 22 and plan:
            continue  # the 4096^2 case runs with the automatic plan only
        with cb.DeviceGrid(a, x, y) as g:
            g.fill_random(c["seed"], thr=np.array(c["thresholds"], dtype=np.uint64))
            g.run(c["steps"], **plan)
            assert g.checksum_str() == c["checksum"], (c, plan)
            if "cells" in c:
                assert (g.cells() == unpack_cells(arrays[c["cells"] + "_out"], a, x, y)).all(), (c, plan)
            assert g.time_step == c["steps"]


def test_random_shapes_and_plans(cuda):
    rng = random.Random(2024)
    for trial in range(120):
        a = rng.randrange(3)
        x = 32 * rng.choice([1, 2, 3, 5, 29, 30, 31, 32, 61, 62, 63, 64, 65, 97])
        y = rng.choice([1, 2, 3, 7, 16, 17, 64, 101])
        steps = rng.randrange(0, 40)
        k, v, lv, r = rng.choice(variants(a))
        plan = dict(temporal_steps=k, words_per_lane=v, levels_per_warp=lv, rows_per_step=r,
                    tile_rows=rng.choice([0, 1, 2, 3, 9, 1000]))
        cells = O.init_cells(x, y, trial, O.thresholds(PROBS[a]))
        got, ck = device_run(a, cells, steps, **plan)
        want = O.run_standard(a, cells, steps)
        assert (got == want).all(), (trial, a, x, y, steps, plan)
        assert ck == O.checksum_str(want)


@pytest.mark.parametrize("automaton", [0, 1, 2])
def test_layout_round_trips(cuda, automaton):
    P = O.PLANES[automaton]
    for (x, y) in [(64, 16), (320, 24), (960, 40)]:
        cells = O.init_cells(x, y, 77, O.thresholds(PROBS[automaton]))
        with cb.DeviceGrid(automaton, x, y) as g:
            g.upload_cells(cells)
            for layout in ("bit_planes", "bit_array", "tiled_bit_planes"):
                for W in (32, 64):
                    try:
                        want = O.pack(layout, cells, P, W)
                    except ValueError:
                        continue
                    if (layout == "bit_planes" and x % W) or (layout == "tiled_bit_planes" and y % (W // 8)):
                        continue
                    img = g.download(layout, W)
                    assert img.data.tobytes() == want.tobytes(), (layout, W)
                    with cb.DeviceGrid(automaton, x, y) as h:
                        h.upload(cb.HostGrid(automaton, layout, W, x, y, want))
                        assert (h.cells() == cells).all(), (layout, W)
            std32 = g.download("standard", 32)
            assert (std32.data.view(np.uint32).reshape(y, x) == cells).all()


def test_layout_runs_match_reference_layout_semantics(cuda):
    # A traverser initialised from a packed layout returns the same layout.
    x, y, steps = 320, 40, 17
    for a in (0, 1, 2):
        P = O.PLANES[a]
        cells = O.init_cells(x, y, 5, O.thresholds(PROBS[a]))
        want = O.run_standard(a, cells, steps)
        for layout, W in (("bit_planes", 64), ("bit_array", 32), ("tiled_bit_planes", 64), ("standard", 8)):
            try:
                img = O.pack(layout, cells, P, W) if layout != "standard" else cells.reshape(-1)
            except ValueError:
                continue
            t = cb.Traverser()
            params = cb.RunParams(automaton=cb.automaton_info(a)[0], x_size=x, y_size=y, steps=steps,
                                  layout=layout, word_size=W, temporal_steps=4)
            t.init(cb.HostGrid(a, layout, W, x, y, img), params)
            t.run(steps)
            out = t.fetch_result()
            assert out.layout == layout
            assert (out.to_standard().cells() == want).all(), (a, layout)


def test_callback_sees_every_chunk(cuda):
    cells = O.init_cells(64, 64, 1, O.thresholds(PROBS[0]))
    seen = []
    t = cb.Traverser()
    t.init(cb.HostGrid.from_cells(0, cells), cb.RunParams(x_size=64, y_size=64, steps=10, temporal_steps=4))
    t.run(10, callback=lambda it, grid: seen.append((it, grid.get_checksum())))
    assert [s[0] for s in seen] == [0, 4, 8, 10]
    for it, ck in seen:
        assert ck == O.checksum_str(O.run_standard(0, cells, it))


def test_invalid_state_is_rejected(cuda):
    cells = np.zeros((8, 32), dtype=np.uint8)
    cells[3, 5] = 2  # game of life has states 0 and 1 only
    with cb.DeviceGrid(0, 32, 8) as g:
        with pytest.raises(cb.StateError, match="State not found"):
            g.upload_cells(cells)


def test_every_variant_on_a_ragged_grid(cuda):
    # 4 strips wide with a ragged last strip, ragged last row tile, wrap on both axes.
    x, y, steps = 32 * 200, 37, 33
    for a in (0, 1, 2):
        cells = O.init_cells(x, y, 1234 + a, O.thresholds(PROBS[a]))
        want = O.run_standard(a, cells, steps)
        for (k, v, lv, r) in variants(a):
            got, _ = device_run(a, cells, steps, temporal_steps=k, words_per_lane=v, levels_per_warp=lv,
                                rows_per_step=r, tile_rows=11)
            assert (got == want).all(), (a, k, v, lv, r)


def test_plan_resolution(cuda):
    p = cb.plan("game-of-life", 65536, 65536, temporal_steps=8, words_per_lane=2, levels_per_warp=4)
    assert (p["temporal_steps"], p["words_per_lane"], p["levels_per_warp"]) == (8, 2, 4)
    assert p["tile_rows"] >= 64
    with pytest.raises(ValueError, match="no strip kernel"):
        cb.plan("game-of-life", 4096, 4096, temporal_steps=2, words_per_lane=4, levels_per_warp=2)
    with pytest.raises(ValueError, match="temporal_steps must be"):
        cb.plan("wire", 4096, 4096, temporal_steps=3)
    with pytest.raises(ValueError, match="rows_per_step must be"):
        cb.plan("wire", 4096, 4096, temporal_steps=16, rows_per_step=3)
    with pytest.raises(ValueError, match="no strip kernel"):
        cb.plan("wire", 4096, 4096, temporal_steps=16, words_per_lane=2, levels_per_warp=2, rows_per_step=4)
    p = cb.plan("excitable", 32768, 32768, temporal_steps=32, words_per_lane=2, levels_per_warp=8, rows_per_step=4)
    assert (p["temporal_steps"], p["levels_per_warp"], p["rows_per_step"]) == (32, 8, 4)
    for a in (0, 1, 2):  # every variant resolves to itself
        for (k, v, lv, r) in variants(a):
            p = cb.plan(a, 8192, 8192, temporal_steps=k, words_per_lane=v, levels_per_warp=lv, rows_per_step=r)
            assert (p["temporal_steps"], p["words_per_lane"], p["levels_per_warp"], p["rows_per_step"]) == (k, v, lv, r)


def test_caller_owned_planes(cuda):
    torch = cuda
    for a in (0, 1, 2):
        x, y, steps = 256, 48, 21
        P = O.PLANES[a]
        cells = O.init_cells(x, y, 9, O.thresholds(PROBS[a]))
        img = O.pack("bit_planes", cells, P, 32)
        buf_a = torch.from_numpy(img.view(np.int32).copy()).cuda()
        buf_b = torch.zeros_like(buf_a)
        plane_bytes = x * y // 8
        pa = [buf_a.data_ptr() + p * plane_bytes for p in range(P)]
        pb = [buf_b.data_ptr() + p * plane_bytes for p in range(P)]
        in_b = cb.run_bit_planes(a, pa, pb, x, y, steps, temporal_steps=4)
        torch.cuda.synchronize()
        res = (buf_b if in_b else buf_a).cpu().numpy().view(np.uint8)
        assert (O.unpack("bit_planes", res, x, y, P, 32) == O.run_standard(a, cells, steps)).all()


def test_gol_4096_against_bit_plane_oracle(cuda):
    x = y = 4096
    steps = 100
    thr = O.thresholds([0.65, 0.35])
    cells = O.init_cells(x, y, 3, thr)
    planes = O.run_bit_planes(0, O.pack("bit_planes", cells, 1, 32).view(np.uint32), x, y, steps)
    with cb.DeviceGrid(0, x, y) as g:
        g.fill_random(3, thr=thr)
        g.run(steps)
        got = g.download("bit_planes", 64)
    assert got.data.tobytes() == planes.view(np.uint8).tobytes()


def test_glider_crosses_the_torus(cuda):
    # A glider moves one cell diagonally every 4 generations: after 4*N
    # generations on an N x N torus it is back where it started.
    for n in (32, 64, 96):
        cells = np.zeros((n, n), dtype=np.uint8)
        for (yy, xx) in [(0, 1), (1, 2), (2, 0), (2, 1), (2, 2)]:
            cells[(yy + 5) % n, (xx + n - 2) % n] = 1  # straddles the x wrap
        for plan in (dict(temporal_steps=8), dict(temporal_steps=1, words_per_lane=1), dict(temporal_steps=16)):
            got, _ = device_run(0, cells, 4 * n, **plan)
            assert (got == cells).all(), (n, plan)
            shifted, _ = device_run(0, cells, 4, **plan)
            assert (shifted == np.roll(cells, (1, 1), axis=(0, 1))).all()


def test_full_size_plans_agree(cuda):
    # Size-independent property at the headline size: every plan computes the
    # same generation (k=1 is the plain one-generation-per-pass schedule).
    x = y = 65536
    thr = cb.thresholds([0.65, 0.35])
    first = None
    sums = []
    for plan in (dict(temporal_steps=8), dict(temporal_steps=1), dict(temporal_steps=4, words_per_lane=1),
                 dict(temporal_steps=16, words_per_lane=4)):
        with cb.DeviceGrid(0, x, y) as g:
            g.fill_random(99, thr=thr)
            g.run(16, **plan)
            sums.append(g.checksum())
            img = g.download("bit_planes", 64).data
            if first is None:
                first = img
            else:
                assert np.array_equal(img, first), plan
    assert all(s == sums[0] for s in sums)
    assert sum(sums[0]) > 0


def test_translation_invariance_large(cuda):
    # Shifting the input toroidally shifts the output (exercises wrap on both
    # axes at a size the scalar oracle cannot reach quickly).
    x, y, steps = 8192, 2048, 24
    for a in (0, 1, 2):
        cells = O.init_cells(x, y, 31, O.thresholds(PROBS[a]))
        base, _ = device_run(a, cells, steps)
        moved, _ = device_run(a, np.roll(cells, (777, 96), axis=(0, 1)), steps)
        assert (np.roll(base, (777, 96), axis=(0, 1)) == moved).all(), a


def test_async_upload_download_pipeline(cuda):
    # cb2_grid_upload_async / cb2_grid_download_async: three grids streamed
    # through two device grids with two copy streams and events, as the
    # bench's e2e leg does, give the synchronous path's results byte for byte.
    torch = cuda
    cases = [(0, 1024, 96, 37), (1, 2048, 64, 21), (2, 512, 160, 50), (0, 1024, 96, 12)]  # the last reuses grid 0
    h2d, d2h, comp = torch.cuda.Stream(), torch.cuda.Stream(), torch.cuda.Stream()
    pinned_in, pinned_out, want = [], [], []
    for i, (a, x, y, steps) in enumerate(cases):
        cells = O.init_cells(x, y, 70 + i, O.thresholds(PROBS[a]))
        n = cb.layout_bytes(a, "bit_planes", 64, x, y)
        pi = torch.empty(n, dtype=torch.uint8, pin_memory=True)
        pi.numpy()[:] = O.pack("bit_planes", cells, O.PLANES[a], 64)
        pinned_in.append(cb.HostGrid(a, "bit_planes", 64, x, y, pi.numpy()))
        pinned_out.append(torch.empty(n, dtype=torch.uint8, pin_memory=True))
        want.append(O.pack("bit_planes", O.run_standard(a, cells, steps), O.PLANES[a], 64))
    slots = {}
    downs = {}
    for i, (a, x, y, steps) in enumerate(cases):
        key = (a, x, y)
        g = slots.setdefault(key, cb.DeviceGrid(a, x, y))
        if key in downs:
            h2d.wait_event(downs[key])
        g.upload_async(pinned_in[i], stream=h2d)
        up = torch.cuda.Event()
        up.record(h2d)
        comp.wait_event(up)
        g.run(steps, stream=comp)
        ran = torch.cuda.Event()
        ran.record(comp)
        d2h.wait_event(ran)
        g.download_async(pinned_out[i].numpy(), stream=d2h)
        downs[key] = torch.cuda.Event()
        downs[key].record(d2h)
    torch.cuda.synchronize()
    for i in range(len(cases)):
        assert pinned_out[i].numpy().tobytes() == want[i].tobytes(), i
    g = next(iter(slots.values()))
    with pytest.raises(ValueError, match="standard"):
        g.upload_async(cb.HostGrid.from_cells(g.automaton, np.zeros((g.y_size, g.x_size), dtype=np.uint8)))
    for g in slots.values():
        g.close()
