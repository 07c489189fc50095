import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "electronphonon.jl_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def gpu_lib():
    """The sm_100a library bound through ctypes; GPU tests fail loudly if it cannot load."""
    import torch

    if not torch.cuda.is_available():
        pytest.fail("GPU test requested but no CUDA device is visible")
    from epb200 import _lib

    return _lib.lib()


@pytest.fixture(scope="session")
def cpu_lib():
    """The library loaded without a GPU, for its host-only entry points."""
    from epb200 import _lib

    return _lib.lib()
