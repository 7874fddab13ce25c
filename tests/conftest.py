import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) CUDA device")


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle
    oracle.build_oracle()
    return oracle
