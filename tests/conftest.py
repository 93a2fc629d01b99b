import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU (B200); parity tests through the C ABI")


def golden(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


@pytest.fixture(scope="session")
def port():
    import oracle

    return oracle.Port()


@pytest.fixture(scope="session")
def kat():
    return {k: float(v) for k, v in np.load(os.path.join(GOLDEN, "kat.npz")).items()}


@pytest.fixture(scope="session")
def port2d():
    import oracle

    return oracle.Fmm2D("port")
