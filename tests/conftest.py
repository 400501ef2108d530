import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs through libmdb200.so")


@pytest.fixture(scope="session")
def built():
    """Builds the library and the oracle once per session."""
    import __graft_entry__

    __graft_entry__.build()
    return True
