"""GPU: evaluation with W and Y in the caller's point order (mxb_plan_set_permutation /
mxb_plan_evaluate_ordered).  The reference permutes W into tree order before its evaluator
(`transform`, matroxTest-V1/hcds.h:766-788) and leaves Y in tree order (matroxTest-V1/Util.h:320);
here split-BF16 plans gather W's rows while splitting W into operand tiles and scatter Y's rows
in the epilogues, FP64 plans permute through leaf-blocked copies.  Every layout (row-major,
column-major, padded leading dimension, column views), both output semantics and every precision
mode must give the leaf-blocked evaluation's numbers, which the oracle pins."""
import numpy as np
import pytest

import oracle as O
from conftest import rel_err
from matrox_ru_b200 import _lib, hgemm as H

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as t
    assert t.cuda.is_available(), "GPU tests need a CUDA device"
    from matrox_ru_b200 import build
    build.build()
    return t


def layouts(torch, A, kind):
    """(N, r) CUDA tensor with A's values in the requested memory layout."""
    t = torch.as_tensor(A, device="cuda")
    if kind == "row":
        return t.contiguous()
    if kind == "col":
        return t.t().contiguous().t()
    if kind == "col_padded":  # column-major with leading dimension N + 13
        buf = torch.full((A.shape[1], A.shape[0] + 13), float("nan"), dtype=torch.float64, device="cuda")
        buf[:, :A.shape[0]] = t.t()
        return buf.t()[:A.shape[0]]
    if kind == "column_view":  # every other column of a row-major (N, 2r) array
        buf = torch.full((A.shape[0], 2 * A.shape[1]), float("nan"), dtype=torch.float64, device="cuda")
        buf[:, ::2] = t
        return buf[:, ::2]
    raise ValueError(kind)


def tree_result(cds, plan, W, r, Y0=None):
    """Leaf-blocked evaluation of the same plan, returned in the caller's order."""
    torch = __import__("torch")
    TW = torch.as_tensor(cds.to_tree_order(W), device="cuda").reshape(-1)
    TY = plan.evaluate(TW, r).cpu().numpy()
    Y = cds.from_tree_order(TY, r)
    return Y if Y0 is None else Y0 + Y


@pytest.mark.parametrize("precision", ["fp64", "split_bf16", "split_bf16_x6", "split_bf16_far6"])
@pytest.mark.parametrize("name", ["h2b", "ragged", "hss"])
def test_ordered_matches_leaf_blocked(torch, small_cases, name, precision):
    cds = small_cases[name]
    r = 200
    rng = np.random.default_rng(21)
    W = rng.standard_normal((cds.n, r))
    Y0 = rng.standard_normal((cds.n, r))
    plan = H.Plan(cds, precision)
    plan.set_permutation(cds.perm)
    want = tree_result(cds, plan, W, r)
    oracle = cds.from_tree_order(O.eval_h2b(cds, cds.to_tree_order(W), r), r)
    tol = 1e-12 if precision == "fp64" else 1e-5
    assert rel_err(want, oracle) <= tol
    for kind in ("row", "col", "col_padded", "column_view"):
        Wt = layouts(torch, W, kind)
        got = plan.evaluate_ordered(Wt).cpu().numpy()
        plan.status()
        assert rel_err(got, want) <= 1e-13, (kind, rel_err(got, want))
        Yt = layouts(torch, Y0, kind)
        plan.evaluate_ordered(Wt, out=Yt, accumulate=True)
        plan.status()
        assert rel_err(Yt.cpu().numpy(), Y0 + want) <= 1e-13, kind
        if kind in ("col_padded", "column_view"):  # nothing outside the view is written
            base = Yt.as_strided((Yt.untyped_storage().nbytes() // 8,), (1,), 0).cpu().numpy()
            assert np.isnan(base).sum() == base.size - Yt.numel()


@pytest.mark.parametrize("nrhs", [1, 130])
def test_ordered_split_column_tails(torch, small_cases, nrhs):
    """One column, and a column count that leaves a partial tile."""
    cds = small_cases["h2b"]
    W = np.random.default_rng(nrhs).standard_normal((cds.n, nrhs))
    plan = H.Plan(cds, "split_bf16")
    plan.set_permutation(cds.perm)
    got = plan.evaluate_ordered(layouts(torch, W, "row")).cpu().numpy()
    plan.status()
    assert rel_err(got, tree_result(cds, plan, W, nrhs)) <= 1e-13


def test_ordered_adjoint_and_evaluator(torch, small_cases):
    cds = small_cases["ragged"]
    r = 17
    rng = np.random.default_rng(3)
    G = rng.standard_normal((cds.n, r))
    ev = H.Evaluator(cds)
    want = cds.from_tree_order(O.adjoint(cds, cds.to_tree_order(G), r), r)
    got = ev.adjoint(torch.as_tensor(G, device="cuda")).cpu().numpy()
    assert rel_err(got, want) <= 1e-12
    W = rng.standard_normal((cds.n, r))
    want = cds.from_tree_order(O.eval_h2b(cds, cds.to_tree_order(W), r), r)
    assert rel_err(ev(torch.as_tensor(W, device="cuda")).cpu().numpy(), want) <= 1e-12


def test_ordered_argument_checks(torch, small_cases):
    cds = small_cases["h2b"]
    plan = H.Plan(cds, "split_bf16")
    W = torch.zeros((cds.n, 8), dtype=torch.float64, device="cuda")
    with pytest.raises(_lib.MxbError) as e:
        plan.evaluate_ordered(W)  # no permutation registered
    assert e.value.code == _lib.MXB_ERR_ARG
    bad = cds.perm.copy()
    bad[0] = bad[1]
    with pytest.raises(_lib.MxbError):
        plan.set_permutation(bad)
    plan.set_permutation(cds.perm)
    with pytest.raises(_lib.MxbError):  # rows alias: stride 0
        plan.evaluate_ordered(torch.zeros(8, dtype=torch.float64, device="cuda").expand(cds.n, 8))
    plan.evaluate_ordered(W)
    plan.status()
