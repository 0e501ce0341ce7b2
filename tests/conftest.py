import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


def _load_golden():
    with open(os.path.join(GOLDEN, "golden.json")) as f:
        meta = json.load(f)
    arrays = np.load(os.path.join(GOLDEN, "golden.npz"))
    return meta["cases"], arrays


@pytest.fixture(scope="session")
def golden():
    return _load_golden()


@pytest.fixture(scope="session")
def cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("GPU test selected but no CUDA device is visible")
    torch.cuda.init()
    return torch
