import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def golden(name):
    return os.path.join(GOLDEN, name)


@pytest.fixture(scope="session")
def awr_cases():
    z = np.load(golden("awr_cases.npz"))
    names = sorted({k[:-2] for k in z.files if k.endswith("_W")})
    out = {}
    for n in names:
        out[n] = {k[len(n) + 1:]: z[k] for k in z.files if k.startswith(n + "_")}
    return out


def cuda_ok():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
