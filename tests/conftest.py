import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); calls the library through its C ABI")


@pytest.fixture(scope="session")
def ora():
    import pyoracle
    pyoracle.lib()
    return pyoracle


@pytest.fixture(scope="session")
def ssp():
    import spec_spars_b200 as S
    S.lib()
    return S


@pytest.fixture(scope="session")
def ctx(ssp):
    c = ssp.Context(0)
    yield c
    c.close()


def rand_graph(n, m, seed, wlo=0.5, whi=2.0):
    """Random simple graph as a symmetric CSC (scipy), seeded."""
    import scipy.sparse as sp
    rng = np.random.default_rng(seed)
    a = rng.integers(0, n, size=3 * m)
    b = rng.integers(0, n, size=3 * m)
    keep = a != b
    a, b = a[keep], b[keep]
    lo, hi = np.minimum(a, b), np.maximum(a, b)
    key = np.unique(lo.astype(np.int64) * n + hi)[:m]
    lo, hi = (key // n).astype(np.int64), (key % n).astype(np.int64)
    w = rng.uniform(wlo, whi, size=len(lo))
    A = sp.coo_matrix((w, (lo, hi)), shape=(n, n))
    A = (A + A.T).tocsc()
    A.sort_indices()
    return A
