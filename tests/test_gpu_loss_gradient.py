"""GPU: the differentiable kernel-ridge loss L = 0.5 ||K~ W - Y||^2 (N = 262144 workload) on an
N = 8192 subsample of its point distribution (d = 18, 32 components, Gaussian h = 1.5,
H2-b budget 0.03, ID tolerance 1e-5, 64 columns, W and Y FP32).  The gradient from the
transposed traversal is checked against central finite differences (exact for a quadratic
loss up to rounding: bar 1e-6) and against the dense K^T G."""
import numpy as np
import pytest

from matrox_ru_b200 import hgemm as H, structure as S
from matrox_ru_b200.autograd import KernelMatVec

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as t
    assert t.cuda.is_available(), "GPU tests need a CUDA device"
    from matrox_ru_b200 import build
    build.build()
    return t


@pytest.fixture(scope="module")
def problem():
    full = S.gaussian_mixture(262144, 18, 32, -2.0, 2.0, 0.3, 1.0, seed=4)
    X = full[np.random.default_rng(5).choice(len(full), 8192, replace=False)]
    spec = S.KernelSpec("gaussian", 1.5)
    cds = S.build_cds(X, spec, leaf_size=256, budget=0.03, tol=1e-5, max_rank=256, seed=6)
    return X, spec, cds


def test_loss_gradient_fd_and_dense(torch, problem):
    X, spec, cds = problem
    ev = H.Evaluator(cds)
    r = 64
    g = torch.Generator(device="cuda").manual_seed(7)
    W = torch.randn(cds.n, r, device="cuda", generator=g, dtype=torch.float32).requires_grad_()
    Yt = torch.randn(cds.n, r, device="cuda", generator=g, dtype=torch.float32)
    loss = 0.5 * ((KernelMatVec.apply(W, ev) - Yt) ** 2).sum()
    loss.backward()
    assert W.grad.dtype == torch.float32 and torch.isfinite(W.grad).all()
    # central differences in FP64 along a random direction
    Wd = W.detach().double()
    V = torch.randn(cds.n, r, device="cuda", generator=g, dtype=torch.float64)
    Yd = Yt.double()
    eps = 1e-3

    def L(w):
        return 0.5 * ((ev(w) - Yd) ** 2).sum().item()

    fd = (L(Wd + eps * V) - L(Wd - eps * V)) / (2 * eps)
    grad64 = ev.adjoint(ev(Wd) - Yd)
    an = (grad64 * V).sum().item()
    assert abs(fd - an) <= 1e-6 * abs(an)
    # FP32 gradient from autograd matches the FP64 gradient to FP32 rounding
    assert (torch.linalg.norm(W.grad.double() - grad64) / torch.linalg.norm(grad64)).item() <= 1e-5
    # dense K^T G on the subsample: the adjoint differs only by the compression error
    G = (ev(Wd) - Yd).cpu().numpy()
    dense = S.dense_kernel_times(X, G, spec)  # K symmetric: K^T G = K G
    rel = np.linalg.norm(grad64.cpu().numpy() - dense) / np.linalg.norm(dense)
    Wn = Wd.cpu().numpy()
    fwd = np.linalg.norm(ev(Wd).cpu().numpy() - S.dense_kernel_times(X, Wn, spec)) / \
        np.linalg.norm(S.dense_kernel_times(X, Wn, spec))
    assert rel <= max(3 * fwd, 1e-3), (rel, fwd)
