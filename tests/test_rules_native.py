"""Host-side check of the word-wide rule networks (cellato_b200/csrc/cb2_rules.cuh):
the same headers, compiled with g++, step random grids one generation at a time
and must match the oracle cell for cell."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "native", "rules_host_check.cpp")


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else shutil.which("g++")
    if not cxx:
        pytest.skip("no host C++ compiler")
    exe = str(tmp_path_factory.mktemp("native") / "rules_host_check")
    subprocess.run([cxx, "-std=c++17", "-O2", SRC, "-o", exe], check=True)
    return exe


@pytest.mark.parametrize("automaton", [0, 1, 2])
def test_networks_match_oracle(checker, automaton):
    probs = {0: [0.5, 0.5], 1: [0.6, 0.05, 0.05, 0.3], 2: [0.125] * 8}[automaton]
    P = O.PLANES[automaton]
    for (x, y, steps, seed) in [(64, 32, 9, 1), (32, 8, 20, 2), (128, 64, 30, 3), (32, 1, 4, 4)]:
        cells = O.init_cells(x, y, seed, O.thresholds(probs))
        packed = O.pack("bit_planes", cells, P, 32)
        out = subprocess.run([checker, str(automaton), str(x), str(y), str(steps)], input=packed.tobytes(),
                             capture_output=True, check=True).stdout
        got = O.unpack("bit_planes", np.frombuffer(out, np.uint8), x, y, P, 32)
        assert (got == O.run_standard(automaton, cells, steps)).all(), (x, y, steps)


def test_pair_networks_exhaustive(checker):
    # the pair evaluation of game-of-life and wire (kernels with two or more rows
    # per step) equals the row-by-row network on every census pattern and centre
    out = subprocess.run([checker, "pairs"], capture_output=True, text=True, check=True).stdout
    assert "game-of-life pairs: 1024 cases, 0 mismatches" in out, out
    assert "wire pairs: 2048 cases, 0 mismatches" in out, out
