import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(REPO, "boundarylayerdynamics.jl_b200")
for p in (os.path.join(REPO, "oracle"), PKG_DIR, REPO):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libbld.so")
    config.addinivalue_line("markers", "slow: long-running CPU test")


def approx(a, b, rtol=None):
    """Julia's ``isapprox`` for arrays: norm(a-b) <= rtol*max(norm(a), norm(b)), rtol = sqrt(eps)."""
    rtol = np.sqrt(np.finfo(float).eps) if rtol is None else rtol
    a = np.asarray(a)
    b = np.asarray(b)
    return bool(np.linalg.norm((a - b).ravel()) <= rtol * max(np.linalg.norm(a.ravel()), np.linalg.norm(b.ravel())))


def rel_l2(a, b):
    a = np.asarray(a).ravel()
    b = np.asarray(b).ravel()
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))


def test_convergence(N, eps, exponential=False, order=None, threshold_linearity=0.99, threshold_slope=0.95):
    """Log-log slope regression (test/test_utils.jl:11-43)."""
    X = np.asarray(N, float) if exponential else np.log(np.asarray(N, float))
    Y = np.log(np.asarray(eps, float))
    n = len(X)
    cov = lambda x, y: np.sum((x - x.mean()) * (y - y.mean())) / (n - 1)
    slope = cov(X, Y) / cov(X, X)
    rsq = cov(X, Y) ** 2 / (cov(X, X) * cov(Y, Y))
    assert rsq > threshold_linearity, (rsq, eps)
    if order is not None:
        assert -slope > order * threshold_slope, (-slope, eps)
    return -slope, rsq


test_convergence.__test__ = False


@pytest.fixture(scope="session")
def oracle():
    import bld_oracle
    return bld_oracle
