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


# One-line reports (FP64 error tables) that GPU tests add with report(); printed
# after the run, so they show in quiet mode too.
_REPORTS: list[str] = []


def report(line: str) -> None:
    _REPORTS.append(line)


def pytest_terminal_summary(terminalreporter, exitstatus, config):
    if _REPORTS:
        terminalreporter.section("error against the FP64 oracle (one step from an identical state)")
        for line in _REPORTS:
            terminalreporter.write_line(line)
