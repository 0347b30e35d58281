import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libsdr_gpu.so")


@pytest.fixture(scope="session")
def golden():
    def load(name):
        return np.load(os.path.join(GOLDEN, name))
    return load


@pytest.fixture(scope="session")
def orc():
    """The oracle restatement (always available: plain C built on demand)."""
    from oracle.oracle import Restatement
    return Restatement()


@pytest.fixture(scope="session")
def ref():
    """The reference's own C build when present, else the restatement."""
    from oracle import oracle
    return oracle.best()


@pytest.fixture(scope="session")
def gpu():
    """The GPU library's python mirror (imports fail loudly without the .so)."""
    from pocketsdr_b200 import sdr_func
    sdr_func.init()
    return sdr_func
