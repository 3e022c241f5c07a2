"""Shared test set-up: import paths, the `gpu` marker, helpers."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "particle-stabilizer_b200", "python")):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


def gpu_available() -> bool:
    try:
        import ctypes

        cudart = ctypes.CDLL("libcuda.so.1")
        n = ctypes.c_int(0)
        if cudart.cuInit(0) != 0:
            return False
        return cudart.cuDeviceGetCount(ctypes.byref(n)) == 0 and n.value > 0
    except OSError:
        return False


@pytest.fixture(scope="session")
def need_gpu():
    if not gpu_available():
        pytest.fail("a CUDA GPU is required for the -m gpu tests")
