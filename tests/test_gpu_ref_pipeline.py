"""GPU: the drop-ins and the plan API on CDSs that the REFERENCE's own host pipeline produced.

Two sources:
* the committed fixtures ``tests/golden/ref_pipeline/*.npz``: the reference's structure
  generator, compression and ``DUV2CDS`` on seeded points, with the outputs of the evaluator
  the generator emitted for that structure (``Y_generated``) and of ``CBHGEMM`` /
  ``parHSSGEMM``;
* the reference pipeline run live (``oracle/_ref/ref_structure`` + ``ref_cds``, built from the
  reference's sources) at the c0 shape (HSS, N=16384, d=8, leaf 128, max rank 128) and the c1
  shape (H2-b, N=65536, d=28, leaf 256, budget 0.03, max rank 256), checked against the
  reference's own ``parHSSGEMM`` / ``CBHGEMM`` on a column slice.

FP64 results must agree with the reference to 1e-12 (relative, max norm); split-BF16 results
stay within 1e-5 (relative, Frobenius) of the FP64 result on the same CDS.
"""
import glob
import os

import numpy as np
import pytest

import oracle as O
import ref_pipeline as RP
from matrox_ru_b200 import _lib, hgemm as H, structure as S

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURES = sorted(glob.glob(os.path.join(HERE, "golden", "ref_pipeline", "*.npz")))
FP64_TOL = 1e-12
SPLIT_TOL = 1e-5


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
    H.set_precision("fp64")
    H.set_flags(0)


def load(path):
    z = np.load(path)
    arrays = {k[4:]: z[k] for k in z.files if k.startswith("cds/")}
    scalars = {k: int(v) for k, v in z["scalars"]}
    return z, RP.cds_from_dump(arrays, scalars), arrays


def rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


def with_reference_offsets(cds, arrays):
    """Make cds.offsets(nrhs) return the reference's own wptr / wskeloffset (written by
    cachewuoffset / coarcacheWUskel for one column; they scale with nrhs)."""
    w1, s1 = arrays["wptr1"].astype(np.int64), arrays["wskeloffset1"].astype(np.int64)
    total1 = int(cds.slen.astype(np.int64).sum())

    def offsets(nrhs):
        w = (w1 * nrhs).astype(np.int32)
        s = (s1 * nrhs).astype(np.int32)
        return w, w.copy(), s, s.copy(), total1 * nrhs
    cds.offsets = offsets
    return cds


H2B_VARIANTS = ["CBHGEMM", "HGEMM", "blockGEMM", "lowH2GEMM"]
HSS_VARIANTS = ["parHSSGEMM", "HGEMM_HSS", "seqHSSGEMM", "lowHSSGEMM"]


@pytest.mark.parametrize("path", FIXTURES, ids=os.path.basename)
def test_dropins_on_the_reference_cds(torch, path):
    """Every drop-in signature on the reference's arrays, against the evaluator the reference
    generated for this structure."""
    z, cds, arrays = load(path)
    r = int(z["nrhs"][0])
    TW, want = z["TW"], z["Y_generated"]
    for variant in (HSS_VARIANTS if cds.is_hss else H2B_VARIANTS):
        apres = np.zeros_like(TW)
        if cds.is_hss:
            H.parHSSGEMM(cds, TW, apres, r, variant=variant)
        else:
            H.CBHGEMM(cds, TW, apres, r, variant=variant)
        assert rel(apres, want) <= FP64_TOL, variant


@pytest.mark.parametrize("path", FIXTURES, ids=os.path.basename)
def test_mirrored_workspaces_at_the_reference_offsets(torch, path):
    """With MXB_FLAG_MIRROR_WORKSPACES the skeleton vectors come back at the caller's offsets;
    at the reference's own offsets they equal what the reference's evaluator leaves there."""
    if not O.ref_available():
        pytest.skip("reference evaluator library not built")
    z, cds, arrays = load(path)
    cds = with_reference_offsets(cds, arrays)
    r = int(z["nrhs"][0])
    ws = O.Workspace(cds, r)
    want = O.eval_h2b(cds, z["TW"], r, use_reference=True, ws=ws)
    wskel = np.full_like(ws.wskel, np.nan)
    uskel = np.zeros_like(ws.uskel)
    apres = np.zeros_like(z["TW"])
    H.set_flags(_lib.FLAG_MIRROR_WORKSPACES)
    (H.parHSSGEMM if cds.is_hss else H.CBHGEMM)(cds, z["TW"], apres, r, wskel=wskel, uskel=uskel)
    assert rel(apres, want) <= FP64_TOL
    assert rel(wskel, ws.wskel) <= FP64_TOL
    assert rel(uskel, ws.uskel) <= FP64_TOL


@pytest.mark.parametrize("path", FIXTURES, ids=os.path.basename)
@pytest.mark.parametrize("precision", ["fp64", "split_bf16"])
def test_plans_on_the_reference_cds(torch, path, precision):
    z, cds, arrays = load(path)
    r = int(z["nrhs"][0])
    plan = H.Plan(cds, precision)
    got = plan.evaluate(torch.as_tensor(z["TW"], device="cuda"), r).cpu().numpy()
    plan.status()
    want = z["Y_generated"]
    if precision == "fp64":
        assert rel(got, want) <= FP64_TOL
    else:
        err = np.linalg.norm(got - want) / np.linalg.norm(want)
        assert 1e-12 < err <= SPLIT_TOL, err


# ---- the reference pipeline run live at the configurations' shapes ----

LIVE = {
    # name: (n, d, components, mean_lo, mean_hi, sigma_lo, sigma_hi, seed, budget, leaf, tol, h, max_rank, nrhs)
    "c0_hss_n16384": (16384, 8, 8, 0.0, 4.0, 0.5, None, 20261202, 0.0, 128, 1e-5, 1.0, 128, 256),
    "c1_h2b_n65536": (65536, 28, 16, -2.0, 2.0, 0.3, 1.0, 20261203, 0.03, 256, 1e-5, 2.0, 256, 1024),
}


@pytest.fixture(scope="module", params=sorted(LIVE))
def live_case(request, tmp_path_factory):
    if not RP.available():
        pytest.skip("reference pipeline binaries not built (oracle/_ref)")
    n, d, k, lo, hi, slo, shi, seed, budget, leaf, tol, h, mr, r = LIVE[request.param]
    X = S.gaussian_mixture(n, d, k, lo, hi, slo, shi, seed=seed)
    run = RP.run(X, budget=budget, leaf=leaf, tol=tol, h=h, max_rank=mr, threads=os.cpu_count() or 1,
                 workdir=str(tmp_path_factory.mktemp(request.param)))
    return request.param, run, r


def leaf_slice(cds, TW, r_full, r):
    out = np.empty(cds.n * r)
    for i in range(cds.nleaf):
        a, b = int(cds.leaf_lids_offset[i]), int(cds.leaf_lids_offset[i + 1])
        out[a * r:b * r] = TW[a * r_full:a * r_full + (b - a) * r]
    return out


def test_live_reference_cds_dropin_and_split(torch, live_case):
    """The generated-evaluator call (HGEMM / HGEMM_HSS with the shape set), then CBHGEMM /
    parHSSGEMM, on all columns of the reference's CDS; a column slice against the reference's
    own evaluator; split-BF16 against FP64 on the same CDS."""
    if not O.ref_available():
        pytest.skip("reference evaluator library not built")
    name, run, r = live_case
    cds = run.cds
    assert cds.is_hss == name.startswith("c0")
    TW = np.random.default_rng(7).standard_normal(cds.n * r)
    first = np.zeros_like(TW)
    if cds.is_hss:
        H.parHSSGEMM(cds, TW, first, r, variant="HGEMM_HSS")
    else:
        H.CBHGEMM(cds, TW, first, r, variant="HGEMM")
    second = np.zeros_like(TW)
    (H.parHSSGEMM if cds.is_hss else H.CBHGEMM)(cds, TW, second, r)
    assert rel(second, first) <= FP64_TOL
    rs = 16
    want = O.eval_h2b(cds, leaf_slice(cds, TW, r, rs), rs, use_reference=True)
    assert rel(leaf_slice(cds, first, r, rs), want) <= FP64_TOL
    plan = H.Plan(cds, "split_bf16")
    got = plan.evaluate(torch.as_tensor(TW, device="cuda"), r).cpu().numpy()
    plan.status()
    err = np.linalg.norm(got - first) / np.linalg.norm(first)
    assert 1e-12 < err <= SPLIT_TOL, err
