import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a); runs on the GPU box")
    config.addinivalue_line("markers", "slow: long-running test")


@pytest.fixture(scope="session")
def golden():
    return np.load(os.path.join(GOLDEN, "contractions.npz"))


@pytest.fixture(scope="session")
def physics():
    with open(os.path.join(GOLDEN, "physics.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def cuda():
    """The CUDA device for -m gpu tests.  The library must be present: no fallback."""
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device in this environment")
    import dmrg_b200

    dmrg_b200.lib()  # raises if libheff_b200.so was not built
    return torch.device("cuda:0")


def relerr(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    nb = np.linalg.norm(b.ravel())
    return float(np.linalg.norm((a - b).ravel()) / (nb if nb > 0 else 1.0))
