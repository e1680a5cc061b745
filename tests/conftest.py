import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the C-ABI library")


def _gpu_present() -> bool:
    try:
        import ctypes
        lib = ctypes.CDLL("libcuda.so.1")
        n = ctypes.c_int(0)
        if lib.cuInit(0) != 0:
            return False
        return lib.cuDeviceGetCount(ctypes.byref(n)) == 0 and n.value > 0
    except OSError:
        return False


GPU = _gpu_present()


@pytest.fixture(scope="session", autouse=True)
def _build_oracle():
    from oracle import oracle
    oracle.build(ref=os.path.isdir(oracle.REF_SRC_DIR))
    yield


@pytest.fixture(scope="session")
def gpu_lib():
    if not GPU:
        pytest.fail("no CUDA device: the gpu tests need a B200")
    from ns3d_wcns_b200 import build
    build.build()
    from ns3d_wcns_b200 import _lib
    return _lib.load()
