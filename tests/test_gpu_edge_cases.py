"""GPU: degenerate shapes against the oracle: a CDS whose tree is a single leaf (the root is the
leaf, so there are no projections, no far couplings and one near block), a four-leaf tree, and
the split-BF16 path at one and at 2048 right-hand sides (16 column tiles of 128)."""
import numpy as np
import pytest

import oracle as O
from conftest import rel_err
from matrox_ru_b200 import hgemm as H, structure as S

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as t
    assert t.cuda.is_available(), "GPU tests need a CUDA device"
    from matrox_ru_b200 import build
    build.build()
    return t


@pytest.fixture(autouse=True)
def _fp64_dropins(torch):
    H.set_precision("fp64")
    H.set_flags(0)
    yield


def tiny(n):
    X = S.gaussian_mixture(n, 3, 2, 0.0, 1.0, 0.3, None, seed=1)
    return S.build_cds(X, S.KernelSpec("gaussian", 1.0), leaf_size=64, budget=0.2, tol=1e-6, max_rank=16)


@pytest.mark.parametrize("n,leaves", [(50, 1), (130, 4)])
def test_tiny_trees_all_paths(torch, n, leaves):
    cds = tiny(n)
    assert cds.nleaf == leaves
    r = 5
    TW = np.random.default_rng(n).standard_normal(cds.n * r)
    want = O.eval_h2b(cds, TW, r)
    tw = torch.as_tensor(TW, device="cuda")
    plan = H.Plan(cds, "fp64")
    assert rel_err(plan.evaluate(tw, r).cpu().numpy(), want) <= 1e-12
    assert rel_err(H.evaluate_host(cds, TW, r), want) <= 1e-12
    assert rel_err(plan.adjoint(tw, r).cpu().numpy(), O.adjoint(cds, TW, r)) <= 1e-12
    split = H.Plan(cds, "split_bf16")
    got = split.evaluate(tw, r).cpu().numpy()
    split.status()
    assert np.linalg.norm(got - want) / np.linalg.norm(want) <= 1e-5


@pytest.mark.parametrize("nrhs", [1, 2048])
def test_split_extreme_nrhs(torch, small_cases, nrhs):
    cds = small_cases["h2b"]
    TW = np.random.default_rng(nrhs).standard_normal(cds.n * nrhs)
    want = O.eval_h2b(cds, TW, nrhs)
    plan = H.Plan(cds, "split_bf16")
    got = plan.evaluate(torch.as_tensor(TW, device="cuda"), nrhs).cpu().numpy()
    plan.status()
    assert 1e-12 < np.linalg.norm(got - want) / np.linalg.norm(want) <= 1e-5


def test_dropin_cache_modes_see_in_place_edits(torch, small_cases):
    """The drop-ins cache the uploaded CDS.  An in-place edit of a value that the default
    (sampled) key does not read is seen after mxb_cache_invalidate, and at once in the
    "full" (every value hashed) and "off" (upload every call) modes."""
    cds = small_cases["h2b"]
    assert cds.D.size >= 2 * 4096  # so the sampled key skips some values
    r = 6
    TW = np.random.default_rng(5).standard_normal(cds.n * r)
    D0 = cds.D.copy()
    try:
        for mode in ("full", "off", "sampled"):
            H.cache_set_mode(mode)
            cds.D[:] = D0
            assert rel_err(H.evaluate_host(cds, TW, r), O.eval_h2b(cds, TW, r)) <= 1e-12
            cds.D[1] += 0.5  # in place: same pointer, same length
            want = O.eval_h2b(cds, TW, r)
            if mode == "sampled":
                H.cache_invalidate()
            assert rel_err(H.evaluate_host(cds, TW, r), want) <= 1e-12, mode
    finally:
        cds.D[:] = D0
        H.cache_set_mode("sampled")
