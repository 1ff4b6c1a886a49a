"""Shared pytest configuration.

Tests marked ``gpu`` need a CUDA device and the built CUDA library.  The
others run on CPU only: the oracle against the golden fixtures, the host-side
logic, and the C-ABI export check.
"""

import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device and the built sm_100a library")


@pytest.fixture(scope="session")
def cuda_device():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda", 0)
