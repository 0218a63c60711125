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
    """The CUDA library on a GPU box; GPU tests fail loudly without it."""
    from dynamics_b200 import _lib
    lib = _lib.lib()
    assert lib.dyn_device_count() > 0, "no CUDA device visible"
    return lib
