import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
HERE = os.path.dirname(os.path.abspath(__file__))
if HERE not in sys.path:
    sys.path.insert(0, HERE)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a); calls the CUDA library")
    config.addinivalue_line("markers", "slow: longer-running case")


@pytest.fixture(scope="session")
def bdg():
    import bdg_lobpcg_b200 as B

    B.lib()
    return B
