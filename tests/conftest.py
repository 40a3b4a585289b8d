"""Test configuration: the `gpu` marker and shared fixtures.

CPU tests (-m "not gpu") cover the oracle against the golden vectors, the
host-side logic and the C-ABI library's exports.  GPU tests call the sm_100a
library through the C ABI and compare with the oracle.
"""
import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test selected but no CUDA device is visible")
    torch.cuda.init()
    return torch.device("cuda:0")


@pytest.fixture(scope="session")
def lib():
    from cholesky_gpu_b200 import _lib
    return _lib.load()
