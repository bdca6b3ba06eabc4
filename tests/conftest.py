import glob
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 (B200) GPU")


def golden(pattern):
    """Golden fixtures (generated by tests/golden/make_golden.py from the reference)."""
    paths = sorted(glob.glob(os.path.join(GOLDEN, pattern + ".npz")))
    assert paths, f"no golden fixture matches {pattern}"
    return [(os.path.basename(p)[:-4], dict(np.load(p))) for p in paths]


def rel(a, b):
    """Normwise relative error ||a-b||_inf / ||b||_inf."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def rel_scaled(a, b, scale):
    """max|a-b| / max(scale): error against the mass of the terms summed into b
    (its floating-point condition scale), for outputs that are differences of
    near-equal sums (the weight gradients)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.max(np.abs(a - b)) / max(float(np.max(np.abs(scale))), 1e-300))


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import OracleLib
    return OracleLib()
