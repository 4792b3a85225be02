import os
import sys

import pytest

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def orc():
    from iga_testlib import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def gold():
    from iga_testlib import golden
    return golden()
