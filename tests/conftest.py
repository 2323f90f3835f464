import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "high-order-regularization_b200")
ORACLE = os.path.join(ROOT, "oracle")
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (ORACLE, PKG, os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 (B200) GPU")


@pytest.fixture(scope="session")
def oracle():
    import build_oracle
    from oracle import Oracle

    build_oracle.build_oracle_lib()
    return Oracle()


@pytest.fixture(scope="session")
def g2s():
    d = np.load(os.path.join(GOLDEN, "ref2s_N16_P4_N0300.npz"))
    return {k: d[k] for k in d.files}


@pytest.fixture(scope="session")
def ge2g():
    d = np.load(os.path.join(GOLDEN, "refe2g_N48.npz"))
    return {k: d[k] for k in d.files}


@pytest.fixture(scope="session")
def ctx():
    import highreg

    c = highreg.Context(0)
    yield c
    c.close()


def rel_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    scale = max(float(np.max(np.abs(b))), 1e-300)
    return float(np.max(np.abs(a - b))) / scale
