"""Shared pytest setup: the `gpu` marker, import paths, and device fixtures."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "fenics-rs_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def fcu():
    """The CUDA library's Python mirror; fails loudly if the .so is missing."""
    import fenics_cuda
    return fenics_cuda


@pytest.fixture(scope="session")
def ctx(fcu):
    c = fcu.Context(0)
    yield c
    c.close()
