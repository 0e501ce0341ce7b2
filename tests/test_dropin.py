"""The C++ drop-in (include/cellato_b200/traverser.hpp) registered as Cellato
suites and driven by the reference's own experiment_manager.  The program is
compiled from the reference headers where they exist (tests/native/Makefile,
run by __graft_entry__.build()) and travels prebuilt."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "cellato_b200", "_build", "dropin_check")
FP_EXE = os.path.join(ROOT, "cellato_b200", "_build", "fingerprint_check")


def test_dropin_binds_configs_by_type_not_name():
    # A config that reuses a registered name with another rule (HighLife as
    # "game-of-life", WireWorld with a reordered dictionary) is rejected by
    # traverser::init before any device call; every bundled config's
    # fingerprint equals the library's.  Needs no GPU.
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "tests", "native")], check=True)
    if not os.path.exists(FP_EXE):
        pytest.skip("neither the reference sources nor a prebuilt fingerprint_check")
    r = subprocess.run([FP_EXE], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "fingerprints ok" in r.stdout
    assert r.stdout.count("rejected:") == 2


def test_dropin_builds_and_fails_cleanly_without_a_gpu():
    # builds where the reference sources exist, keeps a prebuilt binary otherwise
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "tests", "native")], check=True)
    if not os.path.exists(EXE):
        pytest.skip("neither the reference sources nor a prebuilt dropin_check")
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present; the gpu-marked test runs the comparison")
    r = subprocess.run([EXE], capture_output=True, text=True, timeout=120)
    assert r.returncode == 77, r.stdout + r.stderr
    assert "no usable CUDA device" in r.stdout


@pytest.mark.gpu
def test_dropin_matches_reference_cpu_traverser(cuda):
    if not os.path.exists(EXE):
        pytest.skip("dropin_check was not built (the reference sources were absent at build time)")
    r = subprocess.run([EXE], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-4000:] + r.stderr[-2000:]
    assert "all equal" in r.stdout
    assert r.stdout.count(" ok") == 84  # 12 automata x 7 layouts
