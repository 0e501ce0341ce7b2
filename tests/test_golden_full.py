"""The full-size fixtures (tests/golden/full/*.json, from Cellato's own CPU
traverser at the benchmark sizes): their inputs are the oracle's seeded
generator written as bit planes, so the input's checksum and SHA-256 must
follow from the recorded seed and thresholds on the CPU; the GPU test
(test_gpu_full_size.py) compares the device's input and results with them."""
import hashlib
import json
import os

import numpy as np
import pytest

from oracle import oracle as O

FULL = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "full")
NAMES = ["gol-65536", "wire-32768", "excitable-32768"]


@pytest.mark.parametrize("name", NAMES)
def test_full_size_fixture_inputs_follow_from_the_seed(name):
    with open(os.path.join(FULL, f"{name}.json")) as f:
        c = json.load(f)
    assert c["states"].keys() >= {"0", "32", str(c["generations"])}
    thr = np.array(c["thresholds"], dtype=np.uint64)
    assert (thr == O.thresholds(c["probs"])).all()
    planes = O.init_bit_planes(c["x"], c["y"], c["planes"], c["seed"], thr, threads=os.cpu_count() or 1)
    assert hashlib.sha256(planes.view(np.uint8).data).hexdigest() == c["states"]["0"]["sha256"]
    assert "-".join(map(str, O.checksum_planes(planes, c["x"], c["y"], c["planes"]))) == c["states"]["0"]["checksum"]


def test_plane_checksum_and_generator_agree_with_the_cell_forms():
    # orc_checksum_planes / orc_init_bit_planes against orc_checksum / orc_init_cells,
    # including widths whose tiles split words
    for (x, y, P, probs) in [(32, 3, 1, [0.5, 0.5]), (96, 17, 2, [0.6, 0.05, 0.05, 0.3]), (160, 5, 3, [0.125] * 8),
                             (1056, 33, 2, [0.25] * 4)]:
        thr = O.thresholds(probs)
        cells = O.init_cells(x, y, 11, thr)
        planes = O.init_bit_planes(x, y, P, 11, thr, threads=3)
        assert (O.unpack("bit_planes", planes.view(np.uint8), x, y, P, 32) == cells).all()
        assert O.checksum_planes(planes, x, y, P) == O.checksum(cells)
