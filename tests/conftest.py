import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "topo-dda_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libtdda.so")


@pytest.fixture(scope="session")
def sici():
    from oracle import dda_oracle as O

    return O.sici_tables()


@pytest.fixture(scope="session")
def fixture22():
    """The reference's 22x22x10 test structure (python_tests/data), from the
    committed golden fixture."""
    z = np.load(os.path.join(GOLDEN, "fixture_22x22x10.npz"))
    return z
