"""GPU: the FP64 CUDA path against the oracle (parity <= 1e-12 relative, the bar the
FP64 reference mode must meet) through the C-ABI."""
import ctypes
import glob
import os

import numpy as np
import pytest

import oracle as O
from conftest import GOLDEN, rel_err
from matrox_ru_b200 import _lib, hgemm as H, structure as S

pytestmark = pytest.mark.gpu
TOL = 1e-12

FIXTURES = sorted(glob.glob(os.path.join(GOLDEN, "*.npz")))


@pytest.fixture(scope="module")
def torch():
    import torch as t
    assert t.cuda.is_available(), "GPU tests need a CUDA device"
    from matrox_ru_b200 import build
    build.build()
    return t


@pytest.fixture(autouse=True)
def _fp64_mode(torch):
    H.set_precision("fp64")
    H.set_flags(0)
    yield


@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p) for p in FIXTURES])
def test_dropin_matches_reference_golden(torch, path):
    """Reference-signature drop-in on host arrays vs the reference's own outputs."""
    cds = S.CDS.load(path)
    z = np.load(path)
    r = int(z["nrhs"][0])
    apres = z["Y0"].copy()
    H.evaluate_host(cds, z["TW"], r, apres=apres)
    assert rel_err(apres, z["Yref"]) <= TOL


@pytest.mark.parametrize("name", ["hss", "h2b", "ragged"])
@pytest.mark.parametrize("nrhs", [1, 7, 64, 130])
def test_plan_matches_oracle(torch, small_cases, name, nrhs):
    cds = small_cases[name]
    rng = np.random.default_rng(nrhs)
    TW = rng.standard_normal(cds.n * nrhs)
    want = O.eval_h2b(cds, TW, nrhs)
    plan = H.Plan(cds, "fp64")
    got = plan.evaluate(torch.as_tensor(TW, device="cuda"), nrhs)
    torch.cuda.synchronize()
    assert rel_err(got.cpu().numpy(), want) <= TOL


@pytest.mark.parametrize("variant", ["CBHGEMM", "lowH2GEMM", "blockGEMM", "HGEMM"])
def test_h2b_dropin_variants_accumulate(torch, small_cases, variant):
    """H2-b drop-ins accumulate into apres (beta = 1), like the reference."""
    cds = small_cases["h2b"]
    r = 5
    rng = np.random.default_rng(1)
    TW = rng.standard_normal(cds.n * r)
    Y0 = rng.standard_normal(cds.n * r)
    want = O.eval_h2b(cds, TW, r, Y=Y0.copy())
    apres = Y0.copy()
    H.CBHGEMM(cds, TW, apres, r, variant=variant)
    assert rel_err(apres, want) <= TOL


@pytest.mark.parametrize("variant", ["parHSSGEMM", "lowHSSGEMM", "seqHSSGEMM", "HGEMM_HSS"])
def test_hss_dropin_variants_overwrite(torch, small_cases, variant):
    """HSS drop-ins overwrite apres (the reference's HSS near pass has beta = 0)."""
    cds = small_cases["hss"]
    r = 6
    rng = np.random.default_rng(2)
    TW = rng.standard_normal(cds.n * r)
    want = O.eval_h2b(cds, TW, r)
    apres = rng.standard_normal(cds.n * r)  # garbage must be overwritten
    H.parHSSGEMM(cds, TW, apres, r, variant=variant)
    assert rel_err(apres, want) <= TOL


def test_dropin_mirrors_workspaces(torch, small_cases):
    cds = small_cases["h2b"]
    r = 3
    TW = np.random.default_rng(3).standard_normal(cds.n * r)
    ws = O.Workspace(cds, r)
    O.eval_h2b(cds, TW, r, ws=ws)
    wsk = np.zeros_like(ws.wskel)
    usk = np.zeros_like(ws.uskel)
    H.set_flags(_lib.FLAG_MIRROR_WORKSPACES)
    H.CBHGEMM(cds, TW, np.zeros_like(TW), r, wskel=wsk, uskel=usk)
    assert rel_err(wsk, ws.wskel) <= TOL
    assert rel_err(usk, ws.uskel) <= TOL


def test_dropin_cache_reuses_and_invalidates(torch, small_cases):
    cds = small_cases["hss"]
    r = 2
    TW = np.random.default_rng(4).standard_normal(cds.n * r)
    a = H.evaluate_host(cds, TW, r)
    b = H.evaluate_host(cds, TW, r)
    assert np.array_equal(a, b)
    # change a value in place: the sampled checksum may miss it, invalidation must not
    D2 = cds.D.copy()
    cds_mod = S.CDS(**{**cds.__dict__, "D": D2})
    D2 *= 2.0
    H.cache_invalidate()
    c = H.evaluate_host(cds_mod, TW, r)
    assert rel_err(c, O.eval_h2b(cds_mod, TW, r)) <= TOL


@pytest.mark.parametrize("name", ["hss", "h2b", "ragged"])
def test_adjoint_matches_oracle(torch, small_cases, name):
    cds = small_cases[name]
    r = 11
    TG = np.random.default_rng(5).standard_normal(cds.n * r)
    want = O.adjoint(cds, TG, r)
    plan = H.Plan(cds, "fp64")
    got = plan.adjoint(torch.as_tensor(TG, device="cuda"), r)
    assert rel_err(got.cpu().numpy(), want) <= TOL


def test_evaluator_original_order(torch, small_cases):
    """Permutation kernels: (N, r) row-major in point order -> leaf-blocked and back."""
    cds = small_cases["ragged"]
    r = 33
    W = np.random.default_rng(6).standard_normal((cds.n, r))
    ev = H.Evaluator(cds)
    Wt = torch.as_tensor(W, device="cuda")
    TW = ev.to_tree(Wt)
    assert np.array_equal(TW.cpu().numpy(), cds.to_tree_order(W))
    back = ev.from_tree(TW, r)
    assert np.array_equal(back.cpu().numpy(), W)
    Y = ev(Wt).cpu().numpy()
    want = cds.from_tree_order(O.eval_h2b(cds, cds.to_tree_order(W), r), r)
    assert rel_err(Y, want) <= TOL
    # column-major input takes the other stride path
    Wf = torch.as_tensor(np.asfortranarray(W), device="cuda").t().contiguous().t()
    assert rel_err(ev(Wf).cpu().numpy(), want) <= TOL


def test_host_transform_matches_reference_layout(torch, small_cases):
    cds = small_cases["ragged"]
    r = 4
    W = np.random.default_rng(7).standard_normal((cds.n, r))
    TW = H.transform(cds, W, r)
    assert np.array_equal(TW, cds.to_tree_order(W))
    assert np.array_equal(H.untransform(cds, TW, r), W)


def test_autograd_gradient(torch, small_cases):
    from matrox_ru_b200.autograd import KernelMatVec
    cds = small_cases["h2b"]
    ev = H.Evaluator(cds)
    r = 4
    W = torch.randn(cds.n, r, dtype=torch.float64, device="cuda", requires_grad=True)
    T = torch.randn(cds.n, r, dtype=torch.float64, device="cuda")
    loss = 0.5 * ((KernelMatVec.apply(W, ev) - T) ** 2).sum()
    loss.backward()
    Y = ev(W.detach())
    want = ev.adjoint(Y - T)
    assert rel_err(W.grad.cpu().numpy(), want.cpu().numpy()) <= TOL
    # central differences along a random direction
    V = torch.randn_like(W)
    eps = 1e-4
    with torch.no_grad():
        lp = 0.5 * ((ev(W + eps * V) - T) ** 2).sum()
        lm = 0.5 * ((ev(W - eps * V) - T) ** 2).sum()
    fd = (lp - lm) / (2 * eps)
    an = (W.grad * V).sum()
    assert abs(fd.item() - an.item()) <= 1e-6 * abs(an.item())


def test_bad_structure_is_an_error_not_a_fault(torch, small_cases):
    cds = small_cases["h2b"]
    bad = S.CDS(**{**cds.__dict__, "npairy": cds.npairy.copy()})
    bad.npairy[0] = cds.nleaf + 5
    with pytest.raises(_lib.MxbError) as e:
        H.Plan(bad, "fp64")
    assert e.value.code == _lib.MXB_ERR_STRUCTURE
    bad2 = S.CDS(**{**cds.__dict__, "lchildren": cds.lchildren.copy()})
    bad2.lchildren[0] = 0  # self loop
    with pytest.raises(_lib.MxbError):
        H.Plan(bad2, "fp64")


@pytest.mark.skipif(not O.ref_available(), reason="reference library not built")
def test_medium_h2b_vs_reference(torch):
    """A few thousand points, 256 rhs: GPU FP64 vs the reference's CBHGEMM."""
    X = S.gaussian_mixture(8192, 8, 8, 0.0, 4.0, 0.5, None, seed=21)
    cds = S.build_cds(X, S.KernelSpec("gaussian", 2.0), leaf_size=128, budget=0.08, tol=1e-5, max_rank=96)
    r = 256
    TW = np.random.default_rng(8).standard_normal(cds.n * r)
    want = O.eval_h2b(cds, TW, r, use_reference=True)
    plan = H.Plan(cds)
    got = plan.evaluate(torch.as_tensor(TW, device="cuda"), r).cpu().numpy()
    assert rel_err(got, want) <= TOL
