"""Generates the golden fixtures of the lowered DSL automata from Cellato
itself (oracle/_ref/libcellato_ref.so: the reference CPU simple traverser,
standard layout, compiled from the reference headers by oracle/Makefile).

    python tests/golden/make_golden_dsl.py

Covers the bundled automata other than the three with hand-written networks
and the two stochastic examples of include/cellato_b200/dsl_examples.hpp.
Inputs come from the seeded generator (oracle/cellato_oracle.c,
orc_init_cells); each case records the input seed and probabilities, the
run's random seed, the reference checksum, and for small cases the initial
and final cells (uint8 dictionary indexes, golden_dsl.npz).
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402

STATES = {"brian": 3, "critters": 2, "cyclic": 32, "forest-fire": 4, "fluid": 16, "maze": 2, "traffic": 3,
          "lightning-forest": 3, "noisy-life": 2}
PROBS = {"traffic": [0.6, 0.2, 0.2], "lightning-forest": [0.3, 0.6, 0.1], "noisy-life": [0.6, 0.4],
         "maze": [0.7, 0.3], "critters": [0.5, 0.5], "brian": [0.5, 0.2, 0.3]}

# (name, x, y, steps, input seed, run seed, keep cells)
CASES = []
for i, name in enumerate(sorted(STATES)):
    CASES.append((name, 64, 40, 25, 100 + i, 42, True))
    CASES.append((name, 96, 7, 13, 200 + i, 42, True))
    CASES.append((name, 512, 256, 50, 300 + i, 42, False))
for name in ("lightning-forest", "noisy-life"):
    CASES.append((name, 128, 64, 31, 400, 7, True))


def probs_of(name):
    return PROBS.get(name, [1.0 / STATES[name]] * STATES[name])


def main() -> None:
    if not O.ref_available():
        raise SystemExit("oracle/_ref/libcellato_ref.so is missing: run `make -C oracle` with the reference present")
    meta, arrays = [], {}
    for i, (name, x, y, steps, in_seed, run_seed, keep) in enumerate(CASES):
        probs = probs_of(name)
        thr = O.thresholds(probs)
        cells = O.init_cells(x, y, in_seed, thr)
        out, ck = O.ref_run_named(name, cells, steps, seed=run_seed)
        case = {"automaton": name, "x": x, "y": y, "steps": steps, "input_seed": in_seed, "seed": run_seed,
                "probs": probs, "thresholds": [int(t) for t in thr], "checksum": ck}
        if keep:
            arrays[f"d{i}_init"] = cells
            arrays[f"d{i}_out"] = out
            case["cells"] = f"d{i}"
        meta.append(case)
        print(i, name, x, y, steps, ck)
    with open(os.path.join(HERE, "golden_dsl.json"), "w") as f:
        json.dump({"generator": "tests/golden/make_golden_dsl.py", "source": "Cellato CPU simple traverser, "
                   "standard layout (reference headers, oracle/ref_shim.cpp)", "cases": meta}, f, indent=1)
    np.savez_compressed(os.path.join(HERE, "golden_dsl.npz"), **arrays)


if __name__ == "__main__":
    main()
