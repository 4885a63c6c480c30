"""Test configuration.

``-m "not gpu"`` runs everywhere (oracle vs. golden fixtures, host logic,
the C-ABI library's exports, multi-rank host logic on gloo). ``-m gpu``
runs the CUDA path against the oracle and needs a B200.
"""

import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (sm_100a)")


@pytest.fixture(scope="session")
def golden():
    import numpy as np

    def load(name):
        return np.load(GOLDEN / f"{name}.npz")

    return load


@pytest.fixture(scope="session")
def cuda_device():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("a CUDA device is required for gpu-marked tests")
    from quatrex_b200 import build

    build.build()
    return torch.device("cuda", 0)
