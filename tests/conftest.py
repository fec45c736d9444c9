"""Shared test setup.  Tests marked ``gpu`` need a CUDA device (B200) and the built
limbforge_b200 library; everything else runs on the CPU (oracle pinning, host logic, ABI)."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU and the built limbforge_b200 library")


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def golden():
    import numpy as np
    return np.load(os.path.join(ROOT, "tests", "golden", "arith_golden.npz"))


@pytest.fixture(scope="session")
def engine():
    from limbforge_b200 import api
    return api.Engine()
