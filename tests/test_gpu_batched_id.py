"""GPU: the ID compression of the CDS build on the GPU (mxb_batched_id), against the host
restatement of matroxTest-V1/compression.h:446-523 (`decomposition`: LAPACK dgeqp3, the rank
rule |R[s,s] / R[0,0]| < tol capped at max_rank, then the triangular solve for P) on the same
input matrices.  Ranks and skeleton columns must be identical; P agrees to 1e-8 of its largest
entry (the two triangular solves round differently, and R11 can have a condition number near
1 / tol)."""
import numpy as np
import pytest

import oracle as O
from matrox_ru_b200 import hgemm as H, structure as S

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as t
    assert t.cuda.is_available(), "GPU tests need a CUDA device"
    from matrox_ru_b200 import build
    build.build()
    return t


def sample_matrices():
    """Kernel sample matrices shaped like the CDS build's (rows = sampled points, columns =
    candidate points), plus edge cases."""
    rng = np.random.default_rng(7)
    X = S.gaussian_mixture(3000, 6, 5, -2.0, 2.0, 0.3, 1.0, seed=3)
    mats = []
    for nr, nc, kind, h in ((256, 64, "gaussian", 1.0), (512, 256, "gaussian", 2.0), (400, 128, "imq", 1.5),
                            (300, 150, "gaussian", 0.5), (97, 33, "imq", 3.0)):
        idx = rng.choice(X.shape[0], nr + nc, replace=False)
        mats.append(S.kernel_matrix(X, idx[:nr], idx[nr:], S.KernelSpec(kind, h)))
    mats.append(rng.standard_normal((200, 5)) @ rng.standard_normal((5, 60)))  # exact rank 5
    mats.append(np.zeros((40, 12)))                                          # R[0,0] == 0
    mats.append(rng.standard_normal((30, 1)))                                # one column
    mats.append(rng.standard_normal((24, 24)))                               # square
    return mats


@pytest.mark.parametrize("tol,max_rank", [(1e-5, 256), (1e-3, 256), (1e-7, 40)])
def test_batched_id_matches_host_id(torch, tol, max_rank):
    mats = sample_matrices()
    pool = torch.as_tensor(np.concatenate([m.reshape(-1, order="F") for m in mats]), device="cuda")
    got = H.batched_id(pool, [m.shape for m in mats], tol, max_rank)
    for b, (m, (piv, P)) in enumerate(zip(mats, got)):
        hpiv, hP = S.interpolative_decomposition(np.asfortranarray(m), tol, max_rank)
        assert len(piv) == len(hpiv), (b, len(piv), len(hpiv))
        assert np.array_equal(piv, hpiv), b
        assert P.shape == hP.shape
        scale = max(1.0, float(np.abs(hP).max()))
        assert float(np.abs(P - hP).max()) <= 1e-8 * scale, (b, float(np.abs(P - hP).max()))
        # where the tolerance (not max_rank) set the rank, the ID reproduces the matrix to
        # about the tolerance
        if np.abs(m).max() > 0 and len(piv) < min(max_rank, m.shape[1]):
            err = np.linalg.norm(m[:, piv] @ P - m) / np.linalg.norm(m)
            assert err <= 100 * tol + 1e-12, (b, err)
    ranks = [len(p) for p, _ in got]
    assert ranks[5] == 5 and ranks[6] == min(12, max_rank)  # exact rank 5; zero matrix: full
    assert not got[6][1].any()  # zero matrix: P = 0, as in the reference
    if max_rank == 40:
        assert ranks[1] == 40  # capped


def test_batched_id_argument_checks(torch):
    from matrox_ru_b200 import _lib
    pool = torch.zeros(20000, dtype=torch.float64, device="cuda")
    with pytest.raises(_lib.MxbError):
        H.batched_id(pool, [(10, 0)], 1e-5, 8)     # empty matrix
    with pytest.raises(_lib.MxbError):
        H.batched_id(pool, [(10, 10)], 1e-5, 0)    # max_rank < 1
    with pytest.raises(_lib.MxbError) as e:
        H.batched_id(pool, [(2, 9000)], 1e-5, 8)   # more columns than shared memory holds
    assert e.value.code == _lib.MXB_ERR_UNSUPPORTED
    with pytest.raises(ValueError):
        H.batched_id(pool, [(200, 200)], 1e-5, 8)  # pool too small


@pytest.mark.parametrize("name", ["h2b", "hss"])
def test_build_cds_with_gpu_id(torch, name):
    """A CDS built with the GPU ID: the same ranks and skeletons as the host build for nearly
    every node (the GPU's kernel samples differ from the host's in the last bits, which can flip
    a near-tie pivot), the same compression error against the dense K W, and a valid structure
    for the evaluator (FP64 plan vs the oracle on that CDS)."""
    if name == "h2b":
        X = S.gaussian_mixture(768, 4, 4, 0.0, 3.0, 0.4, None, seed=12)
        args = dict(leaf_size=48, budget=0.25, tol=1e-6, max_rank=40)
    else:
        X = S.gaussian_mixture(512, 3, 4, 0.0, 3.0, 0.4, None, seed=11)
        args = dict(leaf_size=32, budget=0.0, tol=1e-6, max_rank=24)
    spec = S.KernelSpec("gaussian", 1.0)
    host = S.build_cds(X, spec, **args)
    gpu = S.build_cds(X, spec, id_on_gpu=True, **args)
    nodes = [v for v in range(1, host.numnodes)]
    same_rank = np.mean([host.slen[v] == gpu.slen[v] for v in nodes])
    same_skel = np.mean([np.array_equal(np.sort(host.skels[v]), np.sort(gpu.skels[v])) for v in nodes])
    assert same_rank >= 0.95 and same_skel >= 0.9, (same_rank, same_skel)
    r = 7
    W = np.random.default_rng(1).standard_normal((X.shape[0], r))
    dense = S.dense_kernel_times(X, W, spec)
    errs = []
    for cds in (host, gpu):
        Y = cds.from_tree_order(O.eval_h2b(cds, cds.to_tree_order(W), r), r)
        errs.append(np.linalg.norm(Y - dense) / np.linalg.norm(dense))
    assert errs[1] <= 2 * errs[0] + 1e-9, errs
    want = O.eval_h2b(gpu, gpu.to_tree_order(W), r)
    got = H.Plan(gpu, "fp64").evaluate(torch.as_tensor(gpu.to_tree_order(W), device="cuda").reshape(-1), r)
    assert np.abs(got.cpu().numpy() - want).max() <= 1e-12 * np.abs(want).max()
