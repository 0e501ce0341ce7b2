"""The DSL golden fixtures (tests/golden/golden_dsl.*, made by
make_golden_dsl.py from the reference CPU traverser): the input generator
reproduces every stored input, and where the reference build is present it
reproduces every stored output and checksum."""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O

HERE = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def golden_dsl():
    with open(os.path.join(HERE, "golden_dsl.json")) as f:
        meta = json.load(f)
    return meta["cases"], np.load(os.path.join(HERE, "golden_dsl.npz"))


def test_inputs_come_from_the_seeded_generator(golden_dsl):
    cases, arrays = golden_dsl
    assert len(cases) >= 20
    for c in cases:
        thr = np.array(c["thresholds"], dtype=np.uint64)
        assert (O.thresholds(c["probs"]) == thr).all()
        if "cells" in c:
            assert (O.init_cells(c["x"], c["y"], c["input_seed"], thr) == arrays[c["cells"] + "_init"]).all()


@pytest.mark.skipif(not O.ref_available(), reason="reference build (oracle/_ref) not present")
def test_the_reference_reproduces_the_fixtures(golden_dsl):
    cases, arrays = golden_dsl
    for c in cases:
        cells = O.init_cells(c["x"], c["y"], c["input_seed"], np.array(c["thresholds"], dtype=np.uint64))
        out, ck = O.ref_run_named(c["automaton"], cells, c["steps"], seed=c["seed"])
        assert ck == c["checksum"], c
        if "cells" in c:
            assert (out == arrays[c["cells"] + "_out"]).all(), c
