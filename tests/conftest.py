import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libtemf_b200.so")
    config.addinivalue_line("markers", "slow: long CPU-oracle runs")


@pytest.fixture(scope="session")
def gpu():
    """A fresh library context on cuda:0 for the test session."""
    from temf3dt_b200.fetd import FetdGPU
    g = FetdGPU(0)
    yield g
    g.close()
