"""GPU: the full H2-b workload (N=65536, d=28, 1024 rhs) through size-independent
properties and a column slice of the reference's own evaluator."""
import numpy as np
import pytest

import oracle as O
from matrox_ru_b200 import _lib, hgemm as H, structure as S

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
def h2b_65536():
    X = S.gaussian_mixture(65536, 28, 16, -2.0, 2.0, 0.3, 1.0, seed=SEED)
    return S.build_cds(X, S.KernelSpec("gaussian", 2.0), leaf_size=256, budget=0.03, tol=1e-5,
                       max_rank=256, seed=SEED)


def leaf_slice(cds, TW, r_full, r):
    out = np.empty(cds.n * r)
    for i in range(cds.nleaf):
        a, b = int(cds.leaf_lids_offset[i]), int(cds.leaf_lids_offset[i + 1])
        out[a * r:b * r] = TW[a * r_full:a * r_full + (b - a) * r]
    return out


def test_h2b_65536_structure_matches_reference_scale(h2b_65536):
    assert (h2b_65536.nleaf, h2b_65536.ncount) == (256, 1536) and 2900 <= h2b_65536.fcount <= 3400
    assert 8.0e11 <= h2b_65536.flops(1024) <= 9.0e11  # the reference's probe at this shape: 8.12e11


def test_h2b_65536_fp64_reference_slice_linearity_and_adjoint(torch, h2b_65536):
    r = 1024
    rng = np.random.default_rng(1)
    W1 = torch.as_tensor(rng.standard_normal(h2b_65536.n * r), device="cuda")
    W2 = torch.as_tensor(rng.standard_normal(h2b_65536.n * r), device="cuda")
    plan = H.Plan(h2b_65536, "fp64")
    Y1 = plan.evaluate(W1, r)
    Y2 = plan.evaluate(W2, r)
    Y12 = plan.evaluate(2.0 * W1 - 0.5 * W2, r)
    lin = (Y12 - (2.0 * Y1 - 0.5 * Y2)).abs().max().item() / Y12.abs().max().item()
    assert lin <= 1e-12
    # the reference's CBHGEMM on the first 8 columns of every leaf block
    if O.ref_available():
        rs = 8
        tw = leaf_slice(h2b_65536, W1.cpu().numpy(), r, rs)
        want = O.eval_h2b(h2b_65536, tw, rs, use_reference=True)
        got = leaf_slice(h2b_65536, Y1.cpu().numpy(), r, rs)
        assert np.abs(got - want).max() / np.abs(want).max() <= 1e-12
    # adjoint identity <K~ W, G> = <W, K~^T G> at full size
    G = torch.as_tensor(rng.standard_normal(h2b_65536.n * r), device="cuda")
    A = plan.adjoint(G, r)
    lhs = torch.dot(Y1, G).item()
    rhs = torch.dot(W1, A).item()
    assert abs(lhs - rhs) <= 1e-10 * abs(lhs)


@pytest.mark.parametrize("mode,tol", [("split_bf16", 1e-5), ("split_bf16_x6", 4e-6)])
def test_h2b_65536_split_bf16_full_columns(torch, h2b_65536, mode, tol):
    r = 1024
    W = torch.as_tensor(np.random.default_rng(2).standard_normal(h2b_65536.n * r), device="cuda")
    want = H.Plan(h2b_65536, "fp64").evaluate(W, r)
    plan = H.Plan(h2b_65536, mode)
    got = plan.evaluate(W, r)
    plan.status()
    err = (torch.linalg.norm(got - want) / torch.linalg.norm(want)).item()
    assert 1e-12 < err <= tol, err


def test_h2b_65536_split_dropin_first_call(torch, h2b_65536):
    """The first drop-in call creates the evaluation graphs of its slab buffers while earlier
    slabs are in flight and the PCIe bus is busy with slab copies: every slab of that call
    must match the plan API on all 1024 columns (the graphs' tables are uploaded in stream
    order, ahead of the launches that read them)."""
    r = 1024
    W = torch.as_tensor(np.random.default_rng(3).standard_normal(h2b_65536.n * r), device="cuda")
    want = H.Plan(h2b_65536, "split_bf16").evaluate(W, r).cpu().numpy()
    tw = torch.empty(h2b_65536.n * r, dtype=torch.float64, pin_memory=True)
    tw.copy_(W.cpu())
    y = torch.zeros(h2b_65536.n * r, dtype=torch.float64, pin_memory=True)
    H.cache_invalidate()
    H.set_precision("split_bf16")
    try:
        for flags in (_lib.FLAG_OUTPUT_IS_ZERO, 0):
            H.set_flags(flags)
            y.zero_()
            H.evaluate_host(h2b_65536, tw.numpy(), r, apres=y.numpy())
            got = y.numpy()
            assert np.abs(got - want).max() <= 1e-6 * np.abs(want).max(), flags
    finally:
        H.set_flags(0)
        H.set_precision("fp64")
        H.cache_invalidate()


@pytest.fixture(scope="module")
def hss_16384():
    """HSS (near-field budget 0): N = 16384 points in d = 8 from an 8-component isotropic
    mixture (means uniform in [0, 4]^8, sigma 0.5), Gaussian h = 1, leaf 128, ID tolerance
    1e-5, max rank 128."""
    X = S.gaussian_mixture(16384, 8, 8, 0.0, 4.0, 0.5, None, seed=SEED)
    spec = S.KernelSpec("gaussian", 1.0)
    return X, spec, S.build_cds(X, spec, leaf_size=128, budget=0.0, tol=1e-5, max_rank=128, seed=SEED)


def test_hss_full_size_vs_reference(torch, hss_16384):
    """The HSS drop-in on all 256 columns against the reference's own parHSSGEMM (FP64,
    <= 1e-12), the split-BF16 path against FP64 (<= 1e-5), and both against the dense K W
    on sampled rows (the compression error, the same for both)."""
    X, spec, cds = hss_16384
    assert cds.is_hss and cds.nleaf == 128
    r = 256
    TW = np.random.default_rng(8).standard_normal(cds.n * r)
    got = H.evaluate_host(cds, TW, r)  # FP64 drop-in (parHSSGEMM signature)
    if O.ref_available():
        want = O.eval_h2b(cds, TW, r, use_reference=True)
        assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()
    plan = H.Plan(cds, "split_bf16")
    split = plan.evaluate(torch.as_tensor(TW, device="cuda"), r).cpu().numpy()
    plan.status()
    assert 1e-12 < np.linalg.norm(split - got) / np.linalg.norm(got) <= 1e-5
    rows = np.random.default_rng(0).choice(cds.n, 64, replace=False)
    dense = S.dense_kernel_times(X, cds.from_tree_order(TW, r), spec, rows=rows)
    e64 = np.linalg.norm(cds.from_tree_order(got, r)[rows] - dense) / np.linalg.norm(dense)
    es = np.linalg.norm(cds.from_tree_order(split, r)[rows] - dense) / np.linalg.norm(dense)
    # HSS compression at max rank 128 leaves ~0.13 here (the ranks saturate); the split path
    # must not add to it beyond its own arithmetic error
    assert e64 < 0.5 and abs(es - e64) <= 1e-5, (e64, es)
