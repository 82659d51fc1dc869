"""GPU: the transposed traversal dGW = K~^T dG on the tensor cores (split-BF16 plans created with
MXB_PLAN_ADJOINT) against the oracle's transposed traversal and the FP64 plan's adjoint.

Bar: relative Frobenius error <= 1e-5 (5e-6 with six products everywhere), well above 1e-12
(the tensor-core kernels ran, not an FP64 kernel).  The adjoint has no counterpart in the
reference; its oracle is the transposed traversal of oracle/hgemm_oracle.c.
"""
import numpy as np
import pytest

import oracle as O
from matrox_ru_b200 import _lib, hgemm as H, structure as S
from matrox_ru_b200.autograd import KernelMatVec

pytestmark = pytest.mark.gpu
TOL = 1e-5


@pytest.fixture(scope="module")
def torch():
    import torch as t
    assert t.cuda.is_available(), "GPU tests need a CUDA device"
    from matrox_ru_b200 import build
    build.build()
    return t


@pytest.fixture(scope="module")
def medium():
    """Ranks near 100-200 and 256-point leaves: several K tiles per item, two row tiles."""
    X = S.gaussian_mixture(4096, 8, 8, 0.0, 4.0, 0.5, None, seed=31)
    return S.build_cds(X, S.KernelSpec("gaussian", 2.0), leaf_size=256, budget=0.2, tol=1e-6, max_rank=200)


def frob(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("mode", ["split_bf16", "split_bf16_far6", "split_bf16_x6"])
@pytest.mark.parametrize("name", ["hss", "h2b", "ragged"])
def test_split_adjoint_matches_oracle(torch, small_cases, name, mode):
    cds = small_cases[name]
    r = 96
    G = np.random.default_rng(5).standard_normal(cds.n * r)
    want = O.adjoint(cds, G, r)
    plan = H.Plan(cds, mode, adjoint=True)
    got = plan.adjoint(torch.as_tensor(G, device="cuda"), r).cpu().numpy()
    plan.status()
    err = frob(got, want)
    assert 1e-12 < err <= (5e-6 if mode == "split_bf16_x6" else TOL), err
    # the forward of the same plan is unchanged by the extra operand tiles
    W = np.random.default_rng(6).standard_normal(cds.n * r)
    y = plan.evaluate(torch.as_tensor(W, device="cuda"), r).cpu().numpy()
    plan.status()
    assert frob(y, O.eval_h2b(cds, W, r)) <= TOL


@pytest.mark.parametrize("nrhs", [1, 130, 300])
def test_split_adjoint_medium_against_fp64_plan(torch, medium, nrhs):
    """Against the FP64 plan's adjoint, several column tiles; then <K~ W, G> = <W, K~^T G> with the
    split forward and the split adjoint of one plan."""
    cds = medium
    rng = np.random.default_rng(nrhs)
    G = torch.as_tensor(rng.standard_normal(cds.n * nrhs), device="cuda")
    W = torch.as_tensor(rng.standard_normal(cds.n * nrhs), device="cuda")
    p64 = H.Plan(cds, "fp64")
    want = p64.adjoint(G, nrhs)
    p64.status()
    sp = H.Plan(cds, "split_bf16", adjoint=True)
    got = sp.adjoint(G, nrhs)
    sp.status()
    err = float(torch.linalg.norm(got - want) / torch.linalg.norm(want))
    assert 1e-12 < err <= TOL, err
    y = sp.evaluate(W, nrhs)
    sp.status()
    lhs, rhs = float(torch.dot(y, G)), float(torch.dot(W, got))
    assert abs(lhs - rhs) <= 1e-5 * (float(torch.linalg.norm(y) * torch.linalg.norm(G))), (lhs, rhs)


def test_split_adjoint_accumulates_and_needs_the_flag(torch, small_cases):
    cds = small_cases["h2b"]
    r = 40
    G = torch.as_tensor(np.random.default_rng(7).standard_normal(cds.n * r), device="cuda")
    plain = H.Plan(cds, "split_bf16")
    with pytest.raises(_lib.MxbError) as e:
        plain.adjoint(G, r)
    assert e.value.code == _lib.MXB_ERR_UNSUPPORTED
    sp = H.Plan(cds, "split_bf16", adjoint=True)
    base = torch.as_tensor(np.random.default_rng(8).standard_normal(cds.n * r), device="cuda")
    out = base.clone()
    sp.adjoint(G, r, out=out, accumulate=True)
    sp.status()
    want = base.cpu().numpy() + O.adjoint(cds, G.cpu().numpy(), r)
    assert frob(out.cpu().numpy(), want) <= TOL


def test_split_adjoint_caller_order_and_autograd(torch, medium):
    """The caller-order adjoint (permuted copies) and the torch.autograd.Function over a
    split-BF16 Evaluator: the gradient of 0.5 ||K~ W - Y||^2 against the FP64 Evaluator's."""
    cds = medium
    r = 64
    rng = np.random.default_rng(9)
    W = torch.as_tensor(rng.standard_normal((cds.n, r)), device="cuda")
    Yt = torch.as_tensor(rng.standard_normal((cds.n, r)), device="cuda")
    grads = {}
    for mode in ("fp64", "split_bf16"):
        ev = H.Evaluator(cds, mode)
        w = W.clone().requires_grad_(True)
        loss = 0.5 * ((KernelMatVec.apply(w, ev) - Yt) ** 2).sum()
        loss.backward()
        ev.plan.status()
        grads[mode] = w.grad.detach()
        g = ev.adjoint(Yt)
        ev.plan.status()
        grads[mode + "_ordered"] = g
    e1 = float(torch.linalg.norm(grads["split_bf16"] - grads["fp64"]) / torch.linalg.norm(grads["fp64"]))
    e2 = float(torch.linalg.norm(grads["split_bf16_ordered"] - grads["fp64_ordered"]) /
               torch.linalg.norm(grads["fp64_ordered"]))
    # the loss gradient composes the split forward's error (in the residual) with the adjoint's
    assert 1e-12 < e1 <= 2 * TOL, e1
    assert 1e-12 < e2 <= TOL, e2
