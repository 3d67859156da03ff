"""Shared fixtures.  GPU tests are marked `gpu`; everything else runs on CPU."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def gpu_available() -> bool:
    try:
        import ctypes
        ctypes.CDLL("libcuda.so.1")
    except OSError:
        return False
    return True


@pytest.fixture(scope="session")
def golden():
    return GOLDEN
