import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libhtcuda.so")


@pytest.fixture(scope="session")
def built():
    """Make sure the CPU oracle (and libhtcuda.so) are built."""
    import __graft_entry__
    __graft_entry__.build()
    return True
