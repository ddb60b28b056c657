import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU and the built libgalpha.so")


@pytest.fixture(scope="session")
def engine():
    import galpha_b200 as G

    e = G.Engine()
    yield e
    e.close()
