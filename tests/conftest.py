import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def native():
    """The in-tree native library, built if missing (nvcc cross-compiles without a GPU)."""
    from subfv_b200 import build, _lib
    build.build()
    return _lib.load()


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import oracle
    oracle.build()
    return oracle.load()


@pytest.fixture(scope="session")
def cuda_ok():
    import ctypes
    n = ctypes.c_int(0)
    try:
        rt = ctypes.CDLL("libcudart.so.12")
    except OSError:
        pytest.skip("libcudart not found")
    if rt.cudaGetDeviceCount(ctypes.byref(n)) != 0 or n.value < 1:
        pytest.fail("marked gpu but no CUDA device is visible")
    return n.value
