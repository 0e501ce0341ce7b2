"""Generates the golden fixtures from Cellato itself (oracle/_ref/libcellato_ref.so,
the reference CPU simple traverser compiled from the reference headers).

    python tests/golden/make_golden.py

Inputs come from the seeded SplitMix64 generator (oracle/cellato_oracle.c,
orc_init_cells), so each case is described by (x, y, seed, probabilities);
the initial grid is stored too, so the generator itself is pinned.  Outputs:
  golden.json  per case: sizes, steps, seed, thresholds, the reference checksum
               string, and for small cases the file key of the packed cells
  golden.npz   bit-packed (numpy.packbits over the uint8 index planes)
               initial and final cells of the small cases
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

PROBS = {
    0: [0.5, 0.5],
    1: [0.60, 0.05, 0.05, 0.30],  # empty, head, tail, conductor (dictionary order)
    2: [0.125] * 8,
}
PROBS_035 = [0.65, 0.35]

# (automaton, x, y, steps, seed, probs, keep_cells)
CASES = [
    (0, 64, 64, 1, 1, PROBS[0], True),
    (0, 64, 64, 8, 1, PROBS[0], True),
    (0, 64, 64, 33, 2, PROBS[0], True),
    (0, 32, 3, 5, 3, PROBS[0], True),
    (0, 96, 17, 19, 4, PROBS_035, True),
    (0, 1024, 1024, 100, 42, PROBS[0], False),
    (0, 4096, 4096, 12, 7, PROBS_035, False),
    (1, 96, 40, 13, 42, PROBS[1], True),
    (1, 256, 128, 50, 5, PROBS[1], True),
    (1, 32, 9, 7, 6, PROBS[1], True),
    (1, 1024, 512, 64, 11, PROBS[1], False),
    (2, 64, 32, 9, 1, PROBS[2], True),
    (2, 320, 64, 40, 9, PROBS[2], True),
    (2, 32, 5, 11, 10, PROBS[2], True),
    (2, 1024, 512, 64, 12, PROBS[2], False),
]


def main() -> None:
    if not O.ref_available():
        raise SystemExit("oracle/_ref/libcellato_ref.so is missing: run `make -C oracle` with the reference present")
    meta, arrays = [], {}
    for i, (a, x, y, steps, seed, probs, keep) in enumerate(CASES):
        thr = O.thresholds(probs)
        cells = O.init_cells(x, y, seed, thr)
        layout = "standard" if x * y <= 1 << 20 else "bit_planes"
        out, ck = O.ref_run(a, cells, steps, layout, 64)
        case = {"automaton": a, "x": x, "y": y, "steps": steps, "seed": seed, "probs": probs,
                "thresholds": [int(t) for t in thr], "checksum": ck,
                "initial_checksum": O.checksum_str(cells), "reference_layout": layout}
        if keep:
            arrays[f"c{i}_init"] = np.packbits(cells.reshape(-1) if a == 0 else
                                               np.unpackbits(cells.reshape(-1, 1), axis=1)[:, -3:].reshape(-1))
            arrays[f"c{i}_out"] = np.packbits(out.reshape(-1) if a == 0 else
                                              np.unpackbits(out.reshape(-1, 1), axis=1)[:, -3:].reshape(-1))
            case["cells"] = f"c{i}"
        meta.append(case)
        print(i, a, x, y, steps, ck)
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py", "source": "Cellato CPU simple traverser "
                   "(reference headers, oracle/ref_shim.cpp)", "cases": meta}, f, indent=1)
    np.savez_compressed(os.path.join(HERE, "golden.npz"), **arrays)


def unpack_cells(packed: np.ndarray, automaton: int, x: int, y: int) -> np.ndarray:
    """Inverse of the packing above: uint8 (y, x) dictionary indexes."""
    n = x * y
    if automaton == 0:
        return np.unpackbits(packed)[:n].reshape(y, x)
    bits = np.unpackbits(packed)[: n * 3].reshape(n, 3)
    return (bits[:, 0] * 4 + bits[:, 1] * 2 + bits[:, 2]).astype(np.uint8).reshape(y, x)


if __name__ == "__main__":
    main()
