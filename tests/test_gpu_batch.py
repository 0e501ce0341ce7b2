"""Batches: many grids of mixed automata, sizes and step counts in one
persistent kernel (graph-replayed), bit-exact against the oracle, equal to
the one-launch-per-grid path, and the bounded-wait failure path."""
import random

import numpy as np
import pytest

import cellato_b200 as cb
from oracle import oracle as O

pytestmark = pytest.mark.gpu

PROBS = {0: [0.5, 0.5], 1: [0.6, 0.05, 0.05, 0.3], 2: [0.125] * 8}


def make_grids(specs, seed0=0):
    grids, cells = [], []
    for i, (a, x, y) in enumerate(specs):
        c = O.init_cells(x, y, seed0 + i, O.thresholds(PROBS[a]))
        g = cb.DeviceGrid(a, x, y)
        g.upload_cells(c)
        grids.append(g)
        cells.append(c)
    return grids, cells


def random_specs(rng, n, max_words=40, max_rows=90):
    return [(rng.randrange(3), 32 * rng.randint(1, max_words), rng.randint(1, max_rows)) for _ in range(n)]


@pytest.mark.parametrize("opts", [dict(), dict(temporal_steps=4, tile_rows=7), dict(temporal_steps=1),
                                  dict(temporal_steps=2, tile_rows=1), dict(temporal_steps=8, tile_rows=1000)])
def test_mixed_batch_matches_oracle(cuda, opts):
    rng = random.Random(11)
    specs = random_specs(rng, 40)
    steps = [rng.randint(0, 45) for _ in specs]
    grids, cells = make_grids(specs)
    with cb.Batch(grids, steps, **opts) as b:
        b.run()
        b.wait()
    for (a, x, y), g, c, s in zip(specs, grids, cells, steps):
        assert (g.cells() == O.run_standard(a, c, s)).all(), (a, x, y, s, opts)
        assert g.time_step == s


def test_narrow_grids_use_exact_wrap_groups(cuda):
    # every width up to 16 words (group geometry), tiny and ragged heights
    specs = [(a, 32 * w, h) for w in range(1, 17) for (a, h) in ((w % 3, 1 + w % 5), ((w + 1) % 3, 37))]
    steps = [5 + (i % 23) for i in range(len(specs))]
    grids, cells = make_grids(specs, 100)
    with cb.Batch(grids, steps) as b:
        b.run()
        b.wait()
    for (a, x, y), g, c, s in zip(specs, grids, cells, steps):
        assert (g.cells() == O.run_standard(a, c, s)).all(), (a, x, y, s)


@pytest.mark.parametrize("opts", [dict(), dict(temporal_steps=4, tile_rows=24), dict(temporal_steps=8, tile_rows=13),
                                  dict(temporal_steps=32, tile_rows=40)])
def test_narrow_last_strips_run_as_row_bands(cuda, opts):
    # widths of 31..75 words: last strips of 1..14 own words run as 2..10 row
    # bands side by side in the warp, wider ones as one strip; heights from a
    # few rows (fewer rows than bands) to several tile rows, with band counts
    # that divide the tile height or not
    specs = [(w % 3, 32 * w, h) for w in range(31, 76) for h in (1 + (w * 7) % 23, 150)]
    steps = [1 + (i * 13) % 40 for i in range(len(specs))]
    grids, cells = make_grids(specs, 300)
    with cb.Batch(grids, steps, **opts) as b:
        b.run()
        b.wait()
    for (a, x, y), g, c, s in zip(specs, grids, cells, steps):
        assert (g.cells() == O.run_standard(a, c, s)).all(), (a, x, y, s, opts)
    for g in grids:
        g.close()


def test_replays_continue_and_match_per_grid_path(cuda):
    rng = random.Random(5)
    specs = random_specs(rng, 24, max_words=70, max_rows=70)
    steps = [rng.randint(1, 30) for _ in specs]
    grids, cells = make_grids(specs, 200)
    twins, _ = make_grids(specs, 200)
    with cb.Batch(grids, steps) as b, cb.Batch(twins, steps) as t:
        for _ in range(3):  # graph replays; odd chunk counts flip the buffers
            b.run()
        b.wait()
        for _ in range(3):
            t.run_per_grid()
        info = b.info()
    assert info["tasks"] > 0 and info["persistent_ctas"] > 0
    for (a, x, y), g, tw, c, s in zip(specs, grids, twins, cells, steps):
        want = O.run_standard(a, c, 3 * s)
        assert (g.cells() == want).all(), (a, x, y, s)
        assert (tw.cells() == want).all()


def test_grid_advanced_outside_the_batch_is_picked_up(cuda):
    specs = [(0, 64, 40), (1, 96, 33), (2, 160, 20)]
    steps = [7, 9, 3]
    grids, cells = make_grids(specs, 300)
    with cb.Batch(grids, steps) as b:
        b.run()
        grids[1].run(5)  # outside the batch
        b.run()
        b.wait()
    for i, ((a, x, y), g, c) in enumerate(zip(specs, grids, cells)):
        total = 2 * steps[i] + (5 if i == 1 else 0)
        assert (g.cells() == O.run_standard(a, c, total)).all(), i


def test_stalled_dependency_times_out_and_the_context_survives(cuda):
    # A task whose dependency nothing satisfies: its bounded wait runs out,
    # the kernel records it and every warp stops; the host sees TimeoutError.
    specs = [(0, 256, 64), (1, 128, 64)]
    grids, cells = make_grids(specs, 400)
    # chunks of 8: two chunks per grid, one task each, so task 3 is grid 1's second chunk
    with cb.Batch(grids, [16, 16], temporal_steps=8, spin_limit=2000, stall_task=3) as b:
        assert b.info()["tasks"] == 4
        b.run()
        with pytest.raises(TimeoutError, match="spin limit"):
            b.wait()
    # the context is still usable
    g, c = make_grids([(2, 64, 16)], 500)
    g[0].run(3)
    assert (g[0].cells() == O.run_standard(2, c[0], 3)).all()
