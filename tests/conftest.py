import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden", "golden_m100.npz")
CASES = ["100_analytic_direct", "100_analytic_gmres", "100_numeric_direct", "100_numeric_gmres"]
QUANTITIES = ["BVec", "XVec", "TRANSVel", "ROTVel", "POS", "ORIENT"]
# F16.8 output: half a unit in the last printed digit, plus floating slack
GOLDEN_ATOL = 5e-9 + 1e-12


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built librigidfibers.so")


@pytest.fixture(scope="session")
def golden():
    return np.load(GOLDEN)


def gpu_available():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False
