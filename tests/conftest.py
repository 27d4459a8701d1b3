import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs on the B200)")
    config.addinivalue_line("markers", "slow: larger CPU cases")


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle
    oracle.lib()  # builds liboracle.so when missing
    return oracle


@pytest.fixture(scope="session")
def cm():
    """The CUDA library binding; GPU tests only."""
    import cumodp_b200
    assert cumodp_b200.is_cuda_enabled(), "no CUDA device visible"
    return cumodp_b200
