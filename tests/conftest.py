import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")
    config.addinivalue_line("markers", "slow: CPU test taking more than a few seconds")


@pytest.fixture(scope="session")
def oracle_built():
    from oracle import build as ob
    ob.build_restatement()
    return True


@pytest.fixture
def rng():
    return np.random.default_rng(12345)


def seeds(rng, count=1):
    return rng.integers(0, 256, (count, 32), dtype=np.uint8)
