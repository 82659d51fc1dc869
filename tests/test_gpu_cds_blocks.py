"""GPU: the CDS's near blocks D and far couplings B generated on the device from the points
(mxb_kernel_blocks) against the host assembly (structure.build_cds, which restates the
reference's Fsubmatrix, matroxTest-V1/compression.h:256-360), for the Gaussian, inverse
multiquadric and 1/r kernels, HSS and H2-b, ragged leaves and the full N = 65536 workload; and
plans built from the device-generated pools against plans built from the host pools."""
import numpy as np
import pytest

import oracle as O
from conftest import rel_err
from matrox_ru_b200 import hgemm as H, structure as S

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as t
    assert t.cuda.is_available(), "GPU tests need a CUDA device"
    from matrox_ru_b200 import build
    build.build()
    return t


def cases():
    X = S.gaussian_mixture(768, 4, 4, 0.0, 3.0, 0.4, None, seed=12)
    yield "h2b-gaussian", X, S.KernelSpec("gaussian", 1.0), dict(leaf_size=48, budget=0.25, tol=1e-6, max_rank=40)
    X = S.gaussian_mixture(700, 5, 6, -1.0, 1.0, 0.3, 0.8, seed=13)
    yield "ragged-imq", X, S.KernelSpec("imq", 1.5), dict(leaf_size=40, budget=0.2, tol=1e-5, max_rank=32)
    X = S.gaussian_mixture(512, 3, 4, 0.0, 3.0, 0.4, None, seed=11)
    yield "hss-newton", X, S.KernelSpec("newton", 1.0), dict(leaf_size=32, budget=0.0, tol=1e-6, max_rank=24)
    X = S.gaussian_mixture(600, 54, 3, -1.0, 1.0, 0.5, None, seed=14)
    yield "h2b-d54", X, S.KernelSpec("gaussian", 3.0), dict(leaf_size=64, budget=0.2, tol=1e-6, max_rank=48)


def max_rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("name,X,spec,kw", list(cases()), ids=[c[0] for c in cases()])
def test_blocks_match_host_assembly(torch, name, X, spec, kw):
    cds = S.build_cds(X, spec, seed=3, **kw)
    D, B = H.kernel_blocks(cds, X, spec)
    torch.cuda.synchronize()
    assert max_rel(D.cpu().numpy()[:cds.D.size], cds.D) <= 1e-12
    if cds.B.size:
        assert max_rel(B.cpu().numpy()[:cds.B.size], cds.B) <= 1e-12
    # a plan built from the device pools evaluates like one built from the host arrays
    r = 33
    TW = np.random.default_rng(0).standard_normal(cds.n * r)
    tw = torch.as_tensor(TW, device="cuda")
    host = H.Plan(cds, "fp64").evaluate(tw, r).cpu().numpy()
    dev = H.Plan(cds, "fp64", pools=(D, B, None)).evaluate(tw, r).cpu().numpy()
    assert rel_err(dev, host) <= 1e-12
    assert rel_err(dev, O.eval_h2b(cds, TW, r)) <= 1e-12


def test_bad_block_lists_are_errors(torch):
    from matrox_ru_b200 import _lib
    X = torch.zeros(10, 3, dtype=torch.float64, device="cuda")
    out = torch.zeros(100, dtype=torch.float64, device="cuda")
    lib = _lib.load()
    ofs = np.array([0, 4, 8], np.int64)
    idx = np.array([0, 1, 2, 3, 4, 5, 6, 12], np.int32)  # 12 is past the 10 points
    r, c, o = np.array([0], np.int32), np.array([1], np.int32), np.array([0], np.uint64)
    P = lambda a: a.ctypes.data
    rc = lib.mxb_kernel_blocks(X.data_ptr(), 10, 3, 0, 1.0, P(ofs), P(idx), 2, P(r), P(c), P(o), 1,
                               out.data_ptr(), 100, None)
    assert rc == _lib.MXB_ERR_STRUCTURE
    idx[7] = 7
    rc = lib.mxb_kernel_blocks(X.data_ptr(), 10, 3, 0, 1.0, P(ofs), P(idx), 2, P(r), P(c), P(o), 1,
                               out.data_ptr(), 10, None)  # a 4 x 4 block does not fit in 10
    assert rc == _lib.MXB_ERR_STRUCTURE
    rc = lib.mxb_kernel_blocks(X.data_ptr(), 10, 3, 0, 1.0, P(ofs), P(idx), 2, P(r), P(c), P(o), 1,
                               out.data_ptr(), 100, None)
    assert rc == _lib.MXB_OK


def test_full_size_blocks(torch):
    """N = 65536, d = 28, Gaussian h = 2 (2.4 GB of blocks): every element against the host
    assembly, and the generation time."""
    X = S.gaussian_mixture(65536, 28, 16, -2.0, 2.0, 0.3, 1.0, seed=20261203)
    spec = S.KernelSpec("gaussian", 2.0)
    cds = S.build_cds(X, spec, leaf_size=256, budget=0.03, tol=1e-5, max_rank=256, seed=20261203)
    D, B = H.kernel_blocks(cds, X, spec)  # first call: allocations, attribute set-up
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    D, B = H.kernel_blocks(cds, X, spec)
    e1.record()
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    for dev, host in ((D, cds.D), (B, cds.B)):
        h = torch.as_tensor(host, device="cuda")
        assert ((dev[:h.numel()] - h).abs().max() / h.abs().max()).item() <= 1e-12
        del h
    gb = (cds.D.size + cds.B.size) * 8 / 1e9
    print(f"GPU CDS blocks: {gb:.2f} GB in {ms:.2f} ms ({gb / ms:.2f} TB/s)")
    assert ms < 1000.0
