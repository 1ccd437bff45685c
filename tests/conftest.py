import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); parity tests of the CUDA path")


@pytest.fixture(scope="session")
def cuda_lib():
    """The CUDA library, built in-tree if missing.  GPU tests use it directly:
    there is no fallback path."""
    from couplb_b200 import build, lib
    build.build()
    return lib.load()
