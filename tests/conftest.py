import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the in-tree sm_100a library")
    config.addinivalue_line("markers", "slow: longer-running test")


def load_golden(case: str):
    with np.load(os.path.join(GOLDEN, f"golden_{case}.npz")) as z:
        return {k: z[k] for k in z.files}


@pytest.fixture(params=["a", "b"], scope="session")
def golden(request):
    g = load_golden(request.param)
    g["case"] = request.param
    return g


def rel(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
