"""Shared pytest configuration.

Tests marked ``gpu`` need a CUDA device and call the product library through
its C ABI; everything else runs on the CPU (the oracle against the reference's
known answers, the host-side logic, and the library's exported symbols).
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libprimus_gpu.so")


@pytest.fixture(scope="session")
def gpu():
    import primus_b200 as P
    if P.device_count() < 1:
        pytest.fail("no CUDA device visible: the gpu tests need a B200")
    return P
