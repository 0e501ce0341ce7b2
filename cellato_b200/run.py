"""Command-line runner with the reference CLI's flags and CSV line.

    python -m cellato_b200.run --automaton game-of-life --device CUDA --traverser b200 \
        --evaluator bit_planes --layout bit_planes --x_size 4096 --y_size 4096 --steps 100 \
        [--word_size 64] [--temporal_steps 8] [--temporal_tile_size_y 0] [--rounds 1] \
        [--warmup_rounds 0] [--seed 42] [--density 0.5 0.5] [--print_csv_header]

Flags, validation messages and the CSV columns follow the reference app
(src/app/main.cpp:159-249, src/app/validation.hpp:173-267,
experiments/experiment_report.hpp:82-96).  The input is the library's seeded
SplitMix64 generator (cb2_grid_fill_random) with per-state probabilities
(--density, dictionary order; default uniform), generated on the device; the
timed region is the traverser's run (CUDA events), like
experiment_manager::time_gpu_run.
"""
from __future__ import annotations

import argparse
import math
import sys
from fractions import Fraction

from . import grid as G
from .traverser import RunParams


def parse(argv):
    ap = argparse.ArgumentParser(prog="python -m cellato_b200.run", description=__doc__.split("\n\n")[0])
    ap.add_argument("--automaton", default="game-of-life")
    ap.add_argument("--device", default="CUDA")
    ap.add_argument("--traverser", default="b200")
    ap.add_argument("--evaluator", default="bit_planes")
    ap.add_argument("--layout", default="bit_planes")
    ap.add_argument("--x_size", type=int, default=0)
    ap.add_argument("--y_size", type=int, default=0)
    ap.add_argument("--steps", type=int, default=0)
    ap.add_argument("--word_size", type=int, default=64)
    ap.add_argument("--temporal_steps", type=int, default=0)
    ap.add_argument("--temporal_tile_size_y", type=int, default=0)
    ap.add_argument("--words_per_lane", type=int, default=0)
    ap.add_argument("--levels_per_warp", type=int, default=0)
    ap.add_argument("--rows_per_step", type=int, default=0)
    ap.add_argument("--rounds", type=int, default=1)
    ap.add_argument("--warmup_rounds", type=int, default=0)
    ap.add_argument("--seed", type=int, default=42)
    ap.add_argument("--density", type=float, nargs="*", default=None)
    ap.add_argument("--print_csv_header", action="store_true")
    return ap.parse_args(argv)


def validate(a) -> None:
    """Raises ValueError with the reference's wording for invalid options."""
    if a.device != "CUDA" or a.traverser != "b200":
        raise ValueError(f"Invalid --device/--traverser {a.device}/{a.traverser}: this backend is CUDA/b200")
    if a.evaluator != a.layout:
        raise ValueError(f"Invalid --evaluator {a.evaluator}: must match --layout {a.layout}")
    if a.layout not in ("standard", "bit_array", "bit_planes", "tiled_bit_planes"):
        raise ValueError(f"Unknown --layout '{a.layout}'")
    if a.automaton not in G.AUTOMATA:
        raise ValueError(f"Unknown --automaton '{a.automaton}'")
    for flag in ("x_size", "y_size"):
        if getattr(a, flag) <= 0:
            raise ValueError(f"Invalid --{flag} {getattr(a, flag)}: must be positive")
    if a.x_size % 32:
        raise ValueError(f"Invalid --x_size {a.x_size}: must be divisible by 32")
    if a.steps < 0:
        raise ValueError(f"Invalid --steps {a.steps}")
    if a.temporal_steps not in (0, 1, 2, 4, 8, 16, 32):
        raise ValueError(f"Invalid --temporal_steps {a.temporal_steps}: use 1, 2, 4, 8, 16 or 32")
    if a.layout != "standard":
        G.layout_bytes(a.automaton, a.layout, a.word_size, a.x_size, a.y_size)


def main(argv=None) -> int:
    a = parse(sys.argv[1:] if argv is None else argv)
    if a.print_csv_header:
        print(RunParams.csv_header() + ",average_time_ms,average_time_per_cell_ps,std_time_ms,"
                                       "rounds_had_same_checksums,checksum")
        return 0
    try:
        validate(a)
    except (ValueError, LookupError) as e:
        print(f"Error: {e}", file=sys.stderr)
        return 1
    import torch

    name, planes, states = G.automaton_info(a.automaton)
    probs = a.density or [Fraction(1, states)] * states
    thr = G.thresholds(probs)
    stream = torch.cuda.current_stream()
    times, checksums = [], []
    for r in range(a.warmup_rounds + a.rounds):
        with G.DeviceGrid(a.automaton, a.x_size, a.y_size) as g:
            g.fill_random(a.seed, thr=thr, stream=stream)
            g.set_seed(a.seed)  # the run's random seed, as run_params::seed is for the reference
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            g.run(a.steps, a.temporal_steps, a.temporal_tile_size_y, a.words_per_lane, a.levels_per_warp,
                  stream=stream, rows_per_step=a.rows_per_step)
            e1.record(stream)
            e1.synchronize()
            if r >= a.warmup_rounds:
                times.append(e0.elapsed_time(e1))
                checksums.append(g.checksum_str(stream=stream))
    params = RunParams(automaton=a.automaton, evaluator=a.evaluator, layout=a.layout, x_size=a.x_size,
                       y_size=a.y_size, steps=a.steps, word_size=a.word_size, temporal_steps=a.temporal_steps,
                       temporal_tile_size_y=a.temporal_tile_size_y, rounds=a.rounds, warmup_rounds=a.warmup_rounds,
                       seed=a.seed)
    mean = sum(times) / len(times)
    std = math.sqrt(sum((t - mean) ** 2 for t in times) / len(times))
    per_cell_ps = mean * 1e9 / (a.x_size * a.y_size) / a.steps if a.steps else 0.0
    same = all(c == checksums[0] for c in checksums)
    print(f"{params.csv_line()},{mean:.6f},{per_cell_ps:.6f},{std:.6f},{'true' if same else 'false'},{checksums[0]}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
