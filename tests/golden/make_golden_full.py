"""Full-size golden checksums from Cellato itself, for the benchmark workloads.

    python tests/golden/make_golden_full.py [NAME ...]     (default: all three)

Each case runs Cellato's own CPU simple traverser with the bit_planes layout
and 64-bit words (oracle/_ref/libcellato_ref.so, ref_run_planes64) over the
seeded input of the GPU benchmark, built directly as bit planes (a standard
grid of 65536^2 enum cells would take 16 GiB).  The reference CPU traverser is
single-threaded: GoL 65536^2 x 1000 takes about 25 minutes, WireWorld and
Greenberg-Hastings 32768^2 x 2000 about as long; separate NAMEs can run as
separate processes.

Per case `tests/golden/full/<NAME>.json` records, for the initial grid and
after each checkpoint generation: the 16-tile checksum (state values summed
with 64-bit arithmetic over 4x4 tiles, memory/standard_grid.hpp:182-218,
computed from the planes by the oracle's orc_checksum_planes) and the SHA-256
of the bit-plane bytes (P planes of Y rows of X/8 bytes, the reference's
bit_planes words on a little-endian host), so a GPU run is compared with the
reference on every cell.
"""
from __future__ import annotations

import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402

# name: (automaton, planes, x, y, generations, seed, state probabilities in dictionary order, checkpoints)
CASES = {
    "gol-65536": (0, 1, 65536, 65536, 1000, 42, [0.65, 0.35], [32, 1000]),
    "wire-32768": (1, 2, 32768, 32768, 2000, 42, [0.60, 0.05, 0.05, 0.30], [32, 2000]),
    "excitable-32768": (2, 3, 32768, 32768, 2000, 42, [0.125] * 8, [32, 2000]),
}


def digest(planes: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(planes).view(np.uint8).data).hexdigest()


def make(name: str) -> dict:
    a, P, x, y, gens, seed, probs, checkpoints = CASES[name]
    thr = O.thresholds(probs)
    t0 = time.time()
    planes = O.init_bit_planes(x, y, P, seed, thr)
    states = {0: {"checksum": "-".join(map(str, O.checksum_planes(planes, x, y, P))), "sha256": digest(planes)}}
    print(f"{name}: input ready in {time.time() - t0:.0f} s", flush=True)
    t1 = time.time()
    final, snaps = O.ref_run_planes64(a, planes, x, y, gens, checkpoints=checkpoints, seed=42,
                                      report_every=max(1, gens // 20))
    ref_s = time.time() - t1
    for g in sorted(snaps):
        states[g] = {"checksum": "-".join(map(str, O.checksum_planes(snaps[g], x, y, P))), "sha256": digest(snaps[g])}
    case = {"name": name, "automaton": a, "planes": P, "x": x, "y": y, "generations": gens, "seed": seed,
            "probs": probs, "thresholds": [int(t) for t in thr],
            "states": {str(g): v for g, v in sorted(states.items())},
            "reference": "Cellato CPU simple traverser, bit_planes layout, 64-bit words (oracle/ref_shim.cpp "
                         "ref_run_planes64)", "reference_seconds": round(ref_s, 1)}
    os.makedirs(os.path.join(HERE, "full"), exist_ok=True)
    with open(os.path.join(HERE, "full", f"{name}.json"), "w") as f:
        json.dump(case, f, indent=1)
    print(f"{name}: done, reference run {ref_s:.0f} s", flush=True)
    return case


def main() -> None:
    if not O.ref_available():
        raise SystemExit("oracle/_ref/libcellato_ref.so is missing: run `make -C oracle` with the reference present")
    for name in sys.argv[1:] or list(CASES):
        make(name)


if __name__ == "__main__":
    main()
