import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libstokes_b200.so")


@pytest.fixture(scope="session")
def oracle():
    from oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def lib():
    """The CUDA library; on a GPU box its absence is an error, not a skip."""
    from erosion_b200 import build
    build.build()
    from erosion_b200 import _lib
    return _lib.load()
