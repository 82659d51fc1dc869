"""CPU: the oracle restatement pinned to the reference's own evaluator."""
import glob
import os

import numpy as np
import pytest

import oracle as O
from conftest import GOLDEN, rel_err
from matrox_ru_b200 import structure as S

FIXTURES = sorted(glob.glob(os.path.join(GOLDEN, "*.npz")))


def load_fixture(path):
    z = np.load(path)
    return S.CDS.load(path), z


@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p) for p in FIXTURES])
def test_oracle_matches_reference_golden(path):
    """The restatement reproduces the outputs the reference's compiled CBHGEMM /
    parHSSGEMM wrote into the fixture (FP64, <= 1e-13 relative)."""
    cds, z = load_fixture(path)
    r = int(z["nrhs"][0])
    Y = O.eval_h2b(cds, z["TW"], r, Y=z["Y0"].copy())
    assert rel_err(Y, z["Yref"]) <= 1e-13


def test_fixture_set_covers_forms():
    kinds = set()
    for p in FIXTURES:
        cds, _ = load_fixture(p)
        kinds.add("hss" if cds.is_hss else "h2b")
        if len(set(cds.Ddim.tolist())) > 1:
            kinds.add("ragged")
    assert kinds == {"hss", "h2b", "ragged"}


@pytest.mark.skipif(not O.ref_available(), reason="reference library not built here")
@pytest.mark.parametrize("name", ["hss", "h2b", "ragged"])
@pytest.mark.parametrize("nrhs", [1, 9])
def test_oracle_matches_reference_live(small_cases, name, nrhs):
    """Same check against the reference library run now, on fresh inputs."""
    cds = small_cases[name]
    rng = np.random.default_rng(nrhs)
    TW = rng.standard_normal(cds.n * nrhs)
    Y0 = np.zeros_like(TW) if cds.is_hss else rng.standard_normal(cds.n * nrhs)
    a = O.eval_h2b(cds, TW, nrhs, Y=Y0.copy())
    b = O.eval_h2b(cds, TW, nrhs, Y=Y0.copy(), use_reference=True)
    assert rel_err(a, b) <= 1e-13


@pytest.mark.skipif(not O.ref_available(), reason="reference library not built here")
def test_reference_variants_agree(small_cases):
    """blockGEMM (uncoarsened level sets) and CBHGEMM give the same result: the schedule
    arrays only order the work."""
    import ctypes
    cds = small_cases["h2b"]
    r = 4
    TW = np.random.default_rng(0).standard_normal(cds.n * r)
    a = O.eval_h2b(cds, TW, r, use_reference=True)
    ws = O.Workspace(cds, r)
    Y = np.zeros_like(TW)
    keep = []

    def k(x, dt=np.int32):
        x = np.ascontiguousarray(x if np.asarray(x).size else np.zeros(1, dt), dtype=dt)
        keep.append(x)
        return x.ctypes.data_as(ctypes.c_void_p)
    rc = O.ref().ref_blockGEMM(
        k(cds.D, np.float64), k(cds.B, np.float64), k(cds.VT, np.float64), k(cds.Dptr, np.uint64),
        k(cds.Bptr, np.uint64), k(cds.VTptr), k(cds.lchildren), k(cds.rchildren), k(cds.levelset), k(cds.idx),
        k(TW, np.float64), Y.ctypes.data_as(ctypes.c_void_p), ctypes.c_int32(r), k(cds.Ddim), k(ws.wptr),
        k(ws.uptr), ws.wskel.ctypes.data_as(ctypes.c_void_p), k(ws.wsko), ws.uskel.ctypes.data_as(ctypes.c_void_p),
        k(ws.usko), k(cds.lm), k(cds.slen), k(cds.nblockset), k(cds.nblocks), k(cds.npairx), k(cds.npairy),
        k(cds.fblockset), k(cds.fblocks), k(cds.fpairx), k(cds.fpairy), ctypes.c_int32(cds.nrow),
        ctypes.c_int32(cds.frow), ctypes.c_int32(cds.depth))
    assert rc == 0
    assert rel_err(Y, a) <= 1e-13


@pytest.mark.parametrize("name", ["hss", "h2b", "ragged"])
def test_adjoint_is_transpose(small_cases, name):
    """<K~ W, G> == <W, K~^T G> and K~^T equals the transpose of the assembled K~."""
    cds = small_cases[name]
    r = 3
    rng = np.random.default_rng(5)
    TW = rng.standard_normal(cds.n * r)
    TG = rng.standard_normal(cds.n * r)
    Y = O.eval_h2b(cds, TW, r)
    A = O.adjoint(cds, TG, r)
    assert abs((Y * TG).sum() - (TW * A).sum()) <= 1e-11 * abs((Y * TG).sum())
    # assemble K~ column by column on a subset and compare with the adjoint's rows
    n = cds.n
    cols = rng.choice(n, size=6, replace=False)
    for c in cols:
        e = np.zeros(n)
        e[c] = 1.0
        Kc = O.eval_h2b(cds, cds.to_tree_order(e[:, None]), 1)  # tree-order column c of K~
        # row c of K~^T G (original order) must equal <K~[:, c], G>
        Gt = cds.from_tree_order(TG, r)
        At = cds.from_tree_order(A, r)
        Kc_orig = cds.from_tree_order(Kc, 1)[:, 0]
        assert np.allclose(At[c], Kc_orig @ Gt, rtol=1e-11, atol=1e-11)


def test_compression_error_small_for_smooth_kernel():
    """With a wide Gaussian the ID compresses well: K~ W close to the dense K W."""
    X = S.gaussian_mixture(1024, 3, 4, 0.0, 2.0, 0.5, None, seed=3)
    spec = S.KernelSpec("gaussian", 3.0)
    cds = S.build_cds(X, spec, leaf_size=64, budget=0.1, tol=1e-7, max_rank=64)
    W = np.random.default_rng(1).standard_normal((1024, 4))
    Y = cds.from_tree_order(O.eval_h2b(cds, cds.to_tree_order(W), 4), 4)
    Yd = S.dense_kernel_times(X, W, spec)
    assert np.linalg.norm(Y - Yd) / np.linalg.norm(Yd) < 1e-5
