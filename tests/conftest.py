import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def gpu_lib():
    """The CUDA library, built in-tree; GPU tests fail loudly if it cannot run."""
    import torch
    from pip_b200 import build, capi
    build.build()
    if not torch.cuda.is_available():
        pytest.fail("GPU test collected on a machine without a CUDA device")
    torch.cuda.init()
    return capi.lib()
