"""Shared fixtures: the in-tree build, the oracle's CPU solve stage, and GPU helpers."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
TESTS = os.path.dirname(os.path.abspath(__file__))
if TESTS not in sys.path:
    sys.path.insert(0, TESTS)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session", autouse=True)
def built():
    from bearing_b200 import build
    build.build_host()
    build.build_oracle()
    if os.path.exists(build.GPU_LIB) or build._stale(build.GPU_LIB, build.GPU_SOURCES):
        try:
            build.build_gpu()
        except RuntimeError:
            if not os.path.exists(build.GPU_LIB):
                raise
    return True
