import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


GOLDEN = os.path.join(ROOT, "tests", "golden")


@pytest.fixture(scope="session")
def small_cases():
    """Small CDSs covering HSS, H2-b and ragged leaf sizes (built once per session)."""
    from matrox_ru_b200 import structure as S
    cases = {}
    X = S.gaussian_mixture(512, 3, 4, 0.0, 3.0, 0.4, None, seed=11)
    cases["hss"] = S.build_cds(X, S.KernelSpec("gaussian", 1.0), leaf_size=32, budget=0.0, tol=1e-6, max_rank=24)
    X = S.gaussian_mixture(768, 4, 4, 0.0, 3.0, 0.4, None, seed=12)
    cases["h2b"] = S.build_cds(X, S.KernelSpec("gaussian", 1.0), leaf_size=48, budget=0.25, tol=1e-6, max_rank=40)
    X = S.gaussian_mixture(700, 5, 6, -1.0, 1.0, 0.3, 0.8, seed=13)
    cases["ragged"] = S.build_cds(X, S.KernelSpec("imq", 1.5), leaf_size=40, budget=0.2, tol=1e-5, max_rank=32)
    return cases


def rel_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))
