import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libscb200.so")


@pytest.fixture(scope="session")
def engine_lib():
    """The built engine library (built on demand; build needs only nvcc)."""
    from superconga_b200 import build
    build.build()
    from superconga_b200 import _lib
    return _lib.load()
