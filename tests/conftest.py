import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: longer CPU-only checks")


@pytest.fixture(scope="session")
def h2o_he():
    """eT's tests/ccsd_gs_energy molecule rebuilt by the oracle front end."""
    from oracle import frontend as fe
    return fe.et_test_system("ccsd_gs_energy")
