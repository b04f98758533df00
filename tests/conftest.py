import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU")


GOLDEN = os.path.join(ROOT, "tests", "golden", "gemm_golden.npz")


@pytest.fixture(scope="session")
def golden():
    return np.load(GOLDEN)


@pytest.fixture(scope="session")
def blx():
    import blasx_b200
    blasx_b200.lib()
    return blasx_b200


@pytest.fixture(scope="session")
def orc():
    import oracle
    oracle.lib()
    return oracle
