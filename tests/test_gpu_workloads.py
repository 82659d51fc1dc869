"""GPU: two workloads at their full sizes.

* Mixed precision across compression tolerances: the H2-b matrix of N = 65536 points in
  d = 28 (16-component mixture, Gaussian h = 2, leaf 256, budget 0.03, max rank 256) built
  at ID tolerances 1e-3, 1e-5 and 1e-7, times 1024 right-hand sides.  The split-BF16 result
  stays within 1e-5 of the FP64 evaluation of the same CDS at every tolerance, and its error
  against the dense FP64 K W (64 sampled rows) differs from the FP64 evaluator's by no more
  than that arithmetic error: the mixed-precision path adds nothing visible to the
  compression error.
* The differentiable kernel-ridge loss L = 0.5 ||K~ W - Y||^2 at N = 262144 points in
  d = 18 (32-component mixture, Gaussian h = 1.5, budget 0.03, tolerance 1e-5), W and Y
  262144 x 64 FP32: the gradient from the transposed traversal agrees with central finite
  differences to 1e-6 relative and satisfies <K~ W, G> = <W, K~^T G>.  (The dense K^T G
  check runs on an N = 8192 subsample in test_gpu_loss_gradient.py.)
"""
import numpy as np
import pytest

from matrox_ru_b200 import hgemm as H, structure as S
from matrox_ru_b200.autograd import KernelMatVec

pytestmark = pytest.mark.gpu
SEED = 20261203


@pytest.fixture(scope="module")
def torch():
    import torch as t
    assert t.cuda.is_available(), "GPU tests need a CUDA device"
    from matrox_ru_b200 import build
    build.build()
    return t


@pytest.fixture(scope="module")
def points_d28():
    return S.gaussian_mixture(65536, 28, 16, -2.0, 2.0, 0.3, 1.0, seed=SEED)


@pytest.mark.parametrize("tol", [1e-3, 1e-5, 1e-7])
def test_split_bf16_across_compression_tolerances(torch, points_d28, tol):
    X = points_d28
    spec = S.KernelSpec("gaussian", 2.0)
    cds = S.build_cds(X, spec, leaf_size=256, budget=0.03, tol=tol, max_rank=256, seed=SEED)
    r = 1024
    g = torch.Generator(device="cuda").manual_seed(11)
    TW = torch.randn(cds.n * r, dtype=torch.float64, device="cuda", generator=g)
    y64 = H.Plan(cds, "fp64").evaluate(TW, r)
    plan = H.Plan(cds, "split_bf16")
    ys = plan.evaluate(TW, r)
    plan.status()
    arith = (torch.linalg.norm(ys - y64) / torch.linalg.norm(y64)).item()
    assert 1e-12 < arith <= 1e-5, arith
    rows = np.random.default_rng(0).choice(cds.n, 64, replace=False)
    Wo = cds.from_tree_order(TW.cpu().numpy(), r)
    dense = S.dense_kernel_times(X, Wo, spec, rows=rows)
    nd = np.linalg.norm(dense)
    e64 = np.linalg.norm(cds.from_tree_order(y64.cpu().numpy(), r)[rows] - dense) / nd
    es = np.linalg.norm(cds.from_tree_order(ys.cpu().numpy(), r)[rows] - dense) / nd
    assert np.isfinite(e64) and abs(es - e64) <= 2e-5, (tol, e64, es)


def test_kernel_ridge_loss_full_size(torch):
    X = S.gaussian_mixture(262144, 18, 32, -2.0, 2.0, 0.3, 1.0, seed=4)
    cds = S.build_cds(X, S.KernelSpec("gaussian", 1.5), leaf_size=256, budget=0.03, tol=1e-5,
                      max_rank=256, seed=6)
    ev = H.Evaluator(cds)
    r = 64
    g = torch.Generator(device="cuda").manual_seed(7)
    W = torch.randn(cds.n, r, device="cuda", generator=g, dtype=torch.float32).requires_grad_()
    Yt = torch.randn(cds.n, r, device="cuda", generator=g, dtype=torch.float32)
    loss = 0.5 * ((KernelMatVec.apply(W, ev) - Yt) ** 2).sum()
    loss.backward()
    assert W.grad.dtype == torch.float32 and torch.isfinite(W.grad).all()
    Wd = W.detach().double()
    Yd = Yt.double()
    V = torch.randn(cds.n, r, device="cuda", generator=g, dtype=torch.float64)
    eps = 1e-2  # L is quadratic in W: central differences are exact up to rounding

    def L(w):
        return 0.5 * ((ev(w) - Yd) ** 2).sum().item()

    fd = (L(Wd + eps * V) - L(Wd - eps * V)) / (2 * eps)
    R = ev(Wd) - Yd
    grad64 = ev.adjoint(R)
    an = (grad64 * V).sum().item()
    assert abs(fd - an) <= 1e-6 * abs(an), (fd, an)
    assert (torch.linalg.norm(W.grad.double() - grad64) / torch.linalg.norm(grad64)).item() <= 1e-5
    # adjoint identity at full size
    lhs = (ev(Wd) * R).sum().item()
    rhs = (Wd * grad64).sum().item()
    assert abs(lhs - rhs) <= 1e-10 * abs(lhs)
