"""The lowered DSL path (cb2_ast.cuh): every bundled Cellato automaton and the
two user-defined examples, advanced by the strip kernels and compared cell
for cell with the reference's own CPU traverser (oracle/_ref, standard
layout) on the same input -- including the stochastic rules, whose draws
must reproduce the reference's counter-based stream.  The ":dsl" twins of
the hand-written networks must agree with those networks."""
import random

import numpy as np
import pytest

import cellato_b200 as cb
from oracle import oracle as O

pytestmark = pytest.mark.gpu

DSL = ["brian", "critters", "cyclic", "forest-fire", "fluid", "maze", "traffic", "lightning-forest", "noisy-life"]
PROBS = {"traffic": [0.6, 0.2, 0.2], "lightning-forest": [0.3, 0.6, 0.1], "noisy-life": [0.6, 0.4],
         "maze": [0.7, 0.3], "critters": [0.5, 0.5], "brian": [0.5, 0.2, 0.3]}


@pytest.fixture(scope="module")
def ref(cuda):
    if not O.ref_available():
        pytest.skip("reference build (oracle/_ref) not present")
    missing = [n for n in DSL if n not in cb.AUTOMATA]
    if missing:
        pytest.fail(f"library built without the lowered DSL automata: {missing}")
    return O


def cells_for(name, x, y, seed):
    _, _, states = cb.automaton_info(name)
    probs = PROBS.get(name, [1.0 / states] * states)
    return O.init_cells(x, y, seed, O.thresholds(probs))


def device_run(name, cells, steps, seed=42, time_step=0, **plan):
    y, x = cells.shape
    with cb.DeviceGrid(name, x, y) as g:
        g.upload_cells(cells)
        g.set_seed(seed)
        g.time_step = time_step
        g.run(steps, **plan)
        return g.cells(), g.checksum_str()


@pytest.mark.parametrize("name", DSL)
def test_default_plan_matches_the_reference(ref, name):
    for (x, y, steps, seed) in [(64, 48, 37, 1), (32 * 37, 61, 20, 2), (96, 7, 9, 3)]:
        cells = cells_for(name, x, y, seed)
        want, want_ck = ref.ref_run_named(name, cells, steps)
        got, ck = device_run(name, cells, steps)
        assert (got == want).all(), (name, x, y, steps)
        assert ck == want_ck, (name, x, y, steps)


@pytest.mark.parametrize("name", DSL)
def test_every_lowered_variant_matches_the_reference(ref, name):
    x, y, steps = 32 * 70, 37, 21  # 2+ strips wide with a ragged last strip, odd height
    cells = cells_for(name, x, y, 11)
    want, _ = ref.ref_run_named(name, cells, steps)
    for (k, v, lv, r) in cb.variants(name):
        got, _ = device_run(name, cells, steps, temporal_steps=k, words_per_lane=v, levels_per_warp=lv,
                            rows_per_step=r, tile_rows=9)
        assert (got == want).all(), (name, k, v, lv, r)


@pytest.mark.parametrize("name", ["lightning-forest", "noisy-life", "critters", "traffic"])
def test_time_and_seed_dependent_rules(ref, name):
    x, y = 256, 65
    cells = cells_for(name, x, y, 5)
    for seed in (42, 7, 123456789):
        want, _ = ref.ref_run_named(name, cells, 33, seed=seed)
        got, _ = device_run(name, cells, 33, seed=seed)
        assert (got == want).all(), (name, seed)
    # generations counted across runs: 12 then 21 more equal one run of 33
    want, _ = ref.ref_run_named(name, cells, 33)
    with cb.DeviceGrid(name, x, y) as g:
        g.upload_cells(cells)
        g.run(12)
        g.run(21)
        assert g.time_step == 33
        assert (g.cells() == want).all()


def test_random_shapes_and_plans(ref):
    rng = random.Random(77)
    for trial in range(40):
        name = rng.choice(DSL)
        x = 32 * rng.choice([1, 2, 3, 31, 32, 33, 64])
        y = rng.choice([1, 2, 3, 8, 17, 40])
        steps = rng.randrange(0, 30)
        k, v, lv, r = rng.choice(cb.variants(name))
        cells = cells_for(name, x, y, trial)
        want, _ = ref.ref_run_named(name, cells, steps)
        got, _ = device_run(name, cells, steps, temporal_steps=k, words_per_lane=v, levels_per_warp=lv,
                            rows_per_step=r, tile_rows=rng.choice([0, 1, 5, 100]))
        assert (got == want).all(), (trial, name, x, y, steps, (k, v, lv, r))


@pytest.mark.parametrize("base", ["game-of-life", "wire", "excitable"])
def test_dsl_twins_equal_the_hand_written_networks(cuda, base):
    x, y, steps = 2048, 1024, 100
    _, _, states = cb.automaton_info(base)
    cells = O.init_cells(x, y, 3, O.thresholds([1.0 / states] * states))
    hand, hand_ck = device_run(base, cells, steps)
    dsl, dsl_ck = device_run(base + ":dsl", cells, steps)
    assert (hand == dsl).all()
    assert hand_ck == dsl_ck


def test_checksum_sums_state_values_not_indexes(ref):
    # forest-fire's dictionary lists (empty, tree, fire, ash) but the enum is
    # (empty, tree, ash, fire): the checksum must sum the enum values
    assert cb.grid.state_values("forest-fire") == [0, 1, 3, 2]
    cells = cells_for("forest-fire", 128, 64, 9)
    want, want_ck = ref.ref_run_named("forest-fire", cells, 15)
    _, ck = device_run("forest-fire", cells, 15)
    assert ck == want_ck


def test_band_pass_without_time_refuses_dsl_automata(cuda):
    from cellato_b200 import _abi
    from cellato_b200.bands import BandGrid, _planes
    import ctypes
    b = BandGrid("brian", 256, 64)
    t = _abi.tuning()
    rc = _abi.lib.cb2_band_pass(b.automaton, _planes(b.bufs[0]), _planes(b.bufs[1]), 256, b.rows_total,
                                b.ghost, 64, 4, ctypes.byref(t), None)
    assert rc == _abi.CB2_EINVAL and "cb2_band_pass_at" in _abi.last_error()


# narrow (exact-wrap row groups), ragged multi-strip, odd heights, tall
BATCH_SHAPES = [(64, 48), (32 * 37, 61), (96, 7), (512, 40), (32 * 70, 37), (320, 130), (32, 3)]


@pytest.mark.parametrize("opts", [{}, {"temporal_steps": 4, "tile_rows": 16}, {"temporal_steps": 2, "tile_rows": 9}])
def test_batch_kernel_runs_dsl_automata(ref, opts):
    # every lowered rule beside two networks in one batch, each grid with its own
    # seed and length (remainder chunks); two runs, so the second continues the
    # generations the device advanced after the first
    rng = random.Random(len(opts))
    names = DSL + ["game-of-life", "wire", "cyclic", "critters"]
    cases = []
    for i, name in enumerate(names):
        x, y = BATCH_SHAPES[i % len(BATCH_SHAPES)]
        # seeds within the reference's int run_params::seed
        cases.append((name, x, y, rng.randrange(1, 40), rng.randrange(1, 1 << 31), cells_for(name, x, y, 100 + i)))
    grids = []
    for name, x, y, steps, seed, cells in cases:
        g = cb.DeviceGrid(name, x, y)
        g.upload_cells(cells)
        g.set_seed(seed)
        grids.append(g)
    with cb.Batch(grids, [c[3] for c in cases], **opts) as b:
        b.run()
        b.wait()
        b.run()
        b.wait()
    for g, (name, x, y, steps, seed, cells) in zip(grids, cases):
        want, want_ck = ref.ref_run_named(name, cells, 2 * steps, seed=seed)
        assert g.time_step == 2 * steps
        assert (g.cells() == want).all(), (name, x, y, steps)
        assert g.checksum_str() == want_ck, name
        g.close()


@pytest.mark.parametrize("name", ["lightning-forest", "critters", "traffic", "noisy-life"])
def test_batch_banded_last_strips_of_lowered_rules(ref, name):
    # widths whose last strip (1..14 words) runs as 2..10 row bands side by side
    # in the warp: stochastic draws (paired or not, by the bands' lane parity),
    # Margolus blocks and the alternating rule must see the same global cells,
    # rows and generations as in one strip; tiles of 16 rows give several bands
    # per tile row, and ragged last tiles
    rng = random.Random(sum(map(ord, name)))
    cases = []
    for i, w in enumerate((31, 33, 38, 44, 46, 61)):
        y = (50, 33, 70, 17, 64, 29)[i]
        cases.append((32 * w, y, rng.randrange(1, 30), rng.randrange(1, 1 << 31), cells_for(name, 32 * w, y, 400 + i)))
    grids = []
    for x, y, steps, seed, cells in cases:
        g = cb.DeviceGrid(name, x, y)
        g.upload_cells(cells)
        g.set_seed(seed)
        grids.append(g)
    with cb.Batch(grids, [c[2] for c in cases], temporal_steps=8, tile_rows=16) as b:
        b.run()
        b.wait()
    for g, (x, y, steps, seed, cells) in zip(grids, cases):
        want, want_ck = ref.ref_run_named(name, cells, steps, seed=seed)
        assert (g.cells() == want).all(), (name, x, y, steps)
        assert g.checksum_str() == want_ck, (name, x, y)
        g.close()


def test_batch_follows_time_and_seed_set_between_runs(ref):
    # a grid re-timed and re-seeded between runs: the next run rebuilds the
    # schedule and must equal the strip kernels from that generation and seed
    names = ["lightning-forest", "critters", "traffic", "noisy-life"]
    grids, cells0 = [], []
    for i, name in enumerate(names):
        c = cells_for(name, 160, 50, i)
        g = cb.DeviceGrid(name, 160, 50)
        g.upload_cells(c)
        grids.append(g)
        cells0.append(c)
    with cb.Batch(grids, [13] * len(grids)) as b:
        b.run()
        b.wait()
        mids = [g.cells() for g in grids]
        for i, g in enumerate(grids):
            g.time_step = 1000 + 7 * i
            g.set_seed(99 + i)
        b.run()
        b.wait()
    for i, (g, name) in enumerate(zip(grids, names)):
        want, _ = device_run(name, mids[i], 13, seed=99 + i, time_step=1000 + 7 * i)
        assert (g.cells() == want).all(), name
        assert g.time_step == 1000 + 7 * i + 13
        g.close()


def test_served_dsl_requests(ref):
    mix = [("cyclic", 96, 40, 17, 1), ("lightning-forest", 64, 64, 25, 2), ("critters", 128, 33, 12, 3),
           ("game-of-life", 64, 64, 30, 4), ("traffic", 96, 48, 40, 5)]
    with cb.Server(chunk_steps=8) as srv:
        jobs = []
        for (name, x, y, steps, seed) in mix:
            cells = cells_for(name, x, y, seed)
            jobs.append((name, cells, steps, seed, srv.submit(name, x, y, steps, cells=cells, want_cells=True)))
        srv.drain(120)
        for name, cells, steps, seed, rid in jobs:
            assert srv.wait(rid)["state"] == "done"
            # a request's random seed is its seed field (0 when it brings its own cells)
            want, _ = ref.ref_run_named(name, cells, steps, seed=0)
            assert (srv.result_cells(rid) == want).all(), name


def test_served_seeded_requests_with_many_states(ref):
    # device-seeded inputs over every state of a 32-state dictionary (31 thresholds in
    # the request), batched with a 3-state stochastic rule: each equals the grid seeded
    # and advanced alone
    from fractions import Fraction
    jobs = [("cyclic", 256, 96, 45, 77, [Fraction(1, 32)] * 32),
            ("lightning-forest", 320, 70, 29, 78, [0.5, 0.25, 0.25]),
            ("cyclic", 64, 40, 13, 79, [Fraction(1, 32)] * 32)]
    with cb.Server(chunk_steps=16) as srv:
        ids = [srv.submit(name, x, y, steps, seed, probs, want_cells=True) for (name, x, y, steps, seed, probs) in jobs]
        srv.drain(120)
        for rid, (name, x, y, steps, seed, probs) in zip(ids, jobs):
            st = srv.wait(rid)
            assert st["state"] == "done", st
            with cb.DeviceGrid(name, x, y) as g:
                g.fill_random(seed, probs)
                cells = g.cells()
            want, want_ck = ref.ref_run_named(name, cells, steps, seed=seed)
            assert (srv.result_cells(rid) == want).all(), name
            assert "-".join(str(v) for v in st["checksum"]) == want_ck, name


def test_golden_fixtures(cuda):
    # committed outputs of the reference traverser: independent of oracle/_ref
    import json
    import os
    here = os.path.join(os.path.dirname(__file__), "golden")
    with open(os.path.join(here, "golden_dsl.json")) as f:
        cases = json.load(f)["cases"]
    arrays = np.load(os.path.join(here, "golden_dsl.npz"))
    for c in cases:
        thr = np.array(c["thresholds"], dtype=np.uint64)
        with cb.DeviceGrid(c["automaton"], c["x"], c["y"]) as g:
            g.fill_random(c["input_seed"], thr=thr)
            g.set_seed(c["seed"])
            g.run(c["steps"])
            assert g.checksum_str() == c["checksum"], c
            if "cells" in c:
                assert (g.cells() == arrays[c["cells"] + "_out"]).all(), c


@pytest.mark.parametrize("name,states", [("brian", 3), ("lightning-forest", 3), ("cyclic", 32)])
def test_cli_runs_dsl_automata(ref, capsys, name, states):
    # the reference-style CLI: device-seeded input (uniform states), the run's seed for the draws
    from fractions import Fraction
    from cellato_b200 import run
    x, y, steps, seed = 128, 40, 21, 17
    assert run.main(["--automaton", name, "--device", "CUDA", "--traverser", "b200", "--x_size", str(x),
                     "--y_size", str(y), "--steps", str(steps), "--seed", str(seed)]) == 0
    line = capsys.readouterr().out.strip().splitlines()[-1]
    cells = O.init_cells(x, y, seed, O.thresholds([Fraction(1, states)] * states))
    _, want_ck = ref.ref_run_named(name, cells, steps, seed=seed)
    assert line.endswith("," + want_ck), line


@pytest.mark.parametrize("name", ["critters", "lightning-forest", "traffic", "cyclic"])
def test_two_bands_equal_the_global_grid(ref, name):
    # Rank r of 2 owns rows [r*B, (r+1)*B); ghost rows are refreshed from the other
    # band before each pass, as exchange_halos does between GPUs.  Margolus blocks
    # and probability draws read global rows and generations across the split.
    import ctypes
    from cellato_b200 import _abi
    from cellato_b200.bands import BandGrid, _planes
    x, rows, steps, seed = 512, 96, 37, 5
    bands = [BandGrid(name, x, rows, rank=r, world=2) for r in range(2)]
    for b in bands:
        b.fill_random(seed, [0.5, 0.25, 0.25] if b.states == 3 else None)
        b.seed = 9
    g, B = bands[0].ghost, bands[0].band
    t = _abi.tuning()
    left, done = steps, 0
    while left > 0:
        k = bands[0].plan_k()
        while k > left:
            k //= 2
        for r, b in enumerate(bands):
            other = bands[1 - r].planes
            b.planes[:, g - k:g, :] = other[:, g + B - k:g + B, :]
            b.planes[:, g + B:g + B + k, :] = other[:, g:g + k, :]
        for b in bands:
            _abi.check(_abi.lib.cb2_band_pass_at(b.automaton, _planes(b.bufs[b.cur]), _planes(b.bufs[1 - b.cur]), x,
                                                 b.rows_total, g, B, k, done, b.seed, b.row0 - g, rows,
                                                 ctypes.byref(t), None))
            b.cur ^= 1
        left -= k
        done += k
    _, _, states = cb.automaton_info(name)
    probs = [0.5, 0.25, 0.25] if states == 3 else [1.0 / states] * states
    cells = O.init_cells(x, rows, seed, O.thresholds(probs))
    want, want_ck = ref.ref_run_named(name, cells, steps, seed=9)
    got = np.concatenate([O.unpack("bit_planes", b.band_planes_host().numpy().view(np.uint8).reshape(-1), x, B,
                                   b.P, 32) for b in bands], axis=0)
    assert (got == want).all()
    sums = [sum(v) for v in zip(*[b.local_checksum() for b in bands])]
    assert "-".join(str(v) for v in sums) == want_ck


def test_band_grid_runs_dsl_automata_alone(ref):
    # one rank: ghost rows from its own band, the generic BandGrid.run path
    from cellato_b200.bands import BandGrid
    x, rows, steps = 256, 80, 29
    b = BandGrid("lightning-forest", x, rows)
    b.fill_random(3, [0.3, 0.6, 0.1])
    b.seed = 11
    b.run(steps)
    cells = O.init_cells(x, rows, 3, O.thresholds([0.3, 0.6, 0.1]))
    want, want_ck = ref.ref_run_named("lightning-forest", cells, steps, seed=11)
    got = O.unpack("bit_planes", b.band_planes_host().numpy().view(np.uint8).reshape(-1), x, rows, b.P, 32)
    assert (got == want).all()
    assert "-".join(str(v) for v in b.checksum()) == want_ck
