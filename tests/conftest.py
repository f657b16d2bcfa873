import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the sm_100a kernels")


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session", autouse=True)
def built_libraries():
    """Both shared libraries must exist (they are built in-tree by build())."""
    from penguin_2_0_b200 import build as b
    from oracle import pyoracle
    if not os.path.exists(b.OUT):
        b.build()
    pyoracle.build()
    yield


@pytest.fixture(scope="session")
def gpu():
    if not _has_gpu():
        pytest.fail("a gpu-marked test ran without a CUDA device")
    return 0
