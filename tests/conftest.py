import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libmechanic_b200.so")
    config.addinivalue_line("markers", "slow: long-running case")


@pytest.fixture(scope="session")
def oracle_lib():
    import oracle
    oracle.lib()
    return oracle


@pytest.fixture(scope="session")
def cuda_lib():
    """libmechanic_b200.so on a machine with a GPU; a missing GPU or library is an error."""
    import ctypes
    from mechanic_b200 import build, physics
    build.build()
    lib = physics.library()
    count = ctypes.c_int(0)
    cudart = ctypes.CDLL("libcudart.so.12")
    rc = cudart.cudaGetDeviceCount(ctypes.byref(count))
    if rc != 0 or count.value == 0:
        pytest.fail("gpu test selected but no CUDA device is visible")
    return lib
