import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libgt.so")


def cuda_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu():
    """The product library on device 0; fails loudly if it cannot run."""
    if not cuda_available():
        pytest.fail("no CUDA device: -m gpu tests need a B200")
    from tracking_optimizations_b200 import _native
    _native.context(0)
    return _native
