import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the sm_100a library")


@pytest.fixture(scope="session")
def orc():
    import oracle
    return oracle.lib()


@pytest.fixture(scope="session")
def gpu():
    import prism_b200
    return prism_b200.lib()
