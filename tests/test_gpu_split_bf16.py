"""GPU: the split-BF16 tensor-core path (tcgen05) against the FP64 oracle on the same CDS.

Bar: relative Frobenius error <= 1e-5 (the accuracy target of the split path), and the
result must differ from FP64 in the way BF16 splitting does (error well above 1e-12), which
shows the tensor-core kernels ran rather than an FP64 kernel.
"""
import numpy as np
import pytest

import oracle as O
from matrox_ru_b200 import _lib, hgemm as H, structure as S

pytestmark = pytest.mark.gpu
TOL = 1e-5


@pytest.fixture(scope="module")
def torch():
    import torch as t
    assert t.cuda.is_available(), "GPU tests need a CUDA device"
    from matrox_ru_b200 import build
    build.build()
    return t


def frob(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def run_plan(torch, cds, r, seed=0, mode="split_bf16"):
    TW = np.random.default_rng(seed).standard_normal(cds.n * r)
    want = O.eval_h2b(cds, TW, r)
    plan = H.Plan(cds, mode)
    got = plan.evaluate(torch.as_tensor(TW, device="cuda"), r)
    plan.status()
    return got.cpu().numpy(), want, plan


def test_split_smallest_first(torch, small_cases):
    got, want, plan = run_plan(torch, small_cases["hss"], 1)
    assert plan.info()["precision"] == _lib.PREC_SPLIT_BF16
    err = frob(got, want)
    assert 1e-12 < err <= TOL, err


@pytest.mark.parametrize("name", ["hss", "h2b", "ragged"])
@pytest.mark.parametrize("nrhs", [3, 128, 300])
def test_split_matches_fp64(torch, small_cases, name, nrhs):
    got, want, _ = run_plan(torch, small_cases[name], nrhs, seed=nrhs)
    err = frob(got, want)
    assert 1e-12 < err <= TOL, err


@pytest.mark.parametrize("mode", ["split_bf16_far6", "split_bf16_x6"])
@pytest.mark.parametrize("name", ["hss", "h2b", "ragged"])
def test_split_modes_with_six_products(torch, small_cases, name, mode):
    """6-product far couplings (and near, for x6): x6 reaches FP32-level error."""
    got, want, _ = run_plan(torch, small_cases[name], 70, seed=1, mode=mode)
    err = frob(got, want)
    assert 1e-12 < err <= (TOL if mode == "split_bf16_far6" else 5e-6), err


def test_split_accumulate_and_repeat(torch, small_cases):
    cds = small_cases["h2b"]
    r = 64
    TW = np.random.default_rng(3).standard_normal(cds.n * r)
    Y0 = np.random.default_rng(4).standard_normal(cds.n * r)
    want = O.eval_h2b(cds, TW, r, Y=Y0.copy())
    plan = H.Plan(cds, "split_bf16")
    tw = torch.as_tensor(TW, device="cuda")
    for _ in range(2):  # the second run reuses every buffer
        out = torch.as_tensor(Y0, device="cuda").clone()
        plan.evaluate(tw, r, out=out, accumulate=True)
        plan.status()
        assert frob(out.cpu().numpy(), want) <= TOL


def test_split_dropin(torch, small_cases):
    cds = small_cases["ragged"]
    r = 40
    TW = np.random.default_rng(5).standard_normal(cds.n * r)
    want = O.eval_h2b(cds, TW, r)
    H.set_precision("split_bf16")
    try:
        got = H.evaluate_host(cds, TW, r)
    finally:
        H.set_precision("fp64")
    assert 1e-12 < frob(got, want) <= TOL


def test_split_medium_ranks(torch):
    """Ranks near 100 and 128-point leaves: several K tiles per item and two row tiles."""
    X = S.gaussian_mixture(4096, 8, 8, 0.0, 4.0, 0.5, None, seed=31)
    cds = S.build_cds(X, S.KernelSpec("gaussian", 2.0), leaf_size=256, budget=0.2, tol=1e-6, max_rank=200)
    got, want, _ = run_plan(torch, cds, 257, seed=9)
    assert frob(got, want) <= TOL
