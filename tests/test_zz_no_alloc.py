"""GPU: mxb_evaluate_noalloc, the entry point for callers that may not allocate device
memory (their framework's allocator owns the GPU, or their steady-state loop must avoid
cudaMalloc / cudaFree), checked against mxb_plan_evaluate through the C-ABI.

This file is collected last on purpose: if it fails, a run stopped at the first failure has
already run every other test.  It builds its own inputs, so it also passes alone in a fresh
process.
"""
import ctypes

import numpy as np
import pytest

from matrox_ru_b200 import _lib, hgemm as H, structure as S

pytestmark = pytest.mark.gpu
TOL = 1e-12  # the FP64 parity bar of the other GPU tests


@pytest.fixture(scope="module")
def torch():
    import torch as t
    assert t.cuda.is_available(), "GPU tests need a CUDA device"
    from matrox_ru_b200 import build
    build.build()
    return t


def _cases():
    X = S.gaussian_mixture(768, 4, 4, 0.0, 3.0, 0.4, None, seed=41)
    yield "h2b", S.build_cds(X, S.KernelSpec("gaussian", 1.0), leaf_size=48, budget=0.25, tol=1e-6, max_rank=40)
    X = S.gaussian_mixture(700, 5, 6, -1.0, 1.0, 0.3, 0.8, seed=42)
    yield "ragged", S.build_cds(X, S.KernelSpec("imq", 1.5), leaf_size=40, budget=0.2, tol=1e-5, max_rank=32)
    X = S.gaussian_mixture(512, 3, 4, 0.0, 3.0, 0.4, None, seed=43)
    yield "hss", S.build_cds(X, S.KernelSpec("gaussian", 1.0), leaf_size=32, budget=0.0, tol=1e-6, max_rank=24)


def _device_desc(torch, cds, keep):
    """CDS description with host index arrays and device numeric pools (caller-owned)."""
    desc = H.cds_desc(cds, keep)
    for name in ("D", "B", "VT"):
        a = getattr(cds, name)
        t = torch.as_tensor(a if a.size else np.zeros(1), device="cuda")
        keep.append(t)
        setattr(desc, name, t.data_ptr())
    return desc


@pytest.mark.parametrize("name,cds", list(_cases()), ids=lambda x: x if isinstance(x, str) else "")
def test_noalloc_matches_plan_on_two_calls(torch, name, cds):
    lib = _lib.load()
    r = 37
    W = torch.as_tensor(np.random.default_rng(1).standard_normal(cds.n * r), device="cuda")
    want = H.Plan(cds, "fp64").evaluate(W, r).cpu().numpy()
    keep = []
    desc = _device_desc(torch, cds, keep)
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        Y = torch.full((cds.n * r,), float("nan"), dtype=torch.float64, device="cuda")
        rc = lib.mxb_evaluate_noalloc(ctypes.byref(desc), W.data_ptr(), Y.data_ptr(), r, 0, stream)
        _lib.check(rc, "mxb_evaluate_noalloc")
        torch.cuda.synchronize()
        got = Y.cpu().numpy()
        err = np.abs(got - want).max() / np.abs(want).max()
        assert err <= TOL, (call, err)
    # accumulate = 1 adds to the output, like the H2-b reference
    Y0 = torch.as_tensor(np.random.default_rng(2).standard_normal(cds.n * r), device="cuda")
    Y = Y0.clone()
    _lib.check(lib.mxb_evaluate_noalloc(ctypes.byref(desc), W.data_ptr(), Y.data_ptr(), r, 1, stream),
               "mxb_evaluate_noalloc")
    torch.cuda.synchronize()
    assert np.abs(Y.cpu().numpy() - (Y0.cpu().numpy() + want)).max() <= TOL * np.abs(want).max() * 4


def test_noalloc_rejects_problems_beyond_the_static_scratch(torch):
    lib = _lib.load()
    name, cds = next(_cases())
    keep = []
    desc = _device_desc(torch, cds, keep)
    r = (32 << 20) // (16 * int(cds.slen.sum())) + 64  # skeleton workspaces alone exceed 32 MiB
    W = torch.zeros(cds.n * r, dtype=torch.float64, device="cuda")
    Y = torch.zeros_like(W)
    rc = lib.mxb_evaluate_noalloc(ctypes.byref(desc), W.data_ptr(), Y.data_ptr(), r, 0,
                                  torch.cuda.current_stream().cuda_stream)
    assert rc == _lib.MXB_ERR_UNSUPPORTED
    assert b"MXB_NOALLOC_SCRATCH_BYTES" in lib.mxb_last_error()


def test_noalloc_rejects_host_pools(torch):
    """A descriptor whose pools are host arrays (as mxb_plan_create accepts) is refused with
    MXB_ERR_ARG before anything is launched."""
    lib = _lib.load()
    name, cds = next(_cases())
    keep = []
    desc = H.cds_desc(cds, keep)  # D / B / VT left as host arrays
    r = 4
    W = torch.zeros(cds.n * r, dtype=torch.float64, device="cuda")
    Y = torch.zeros_like(W)
    rc = lib.mxb_evaluate_noalloc(ctypes.byref(desc), W.data_ptr(), Y.data_ptr(), r, 0,
                                  torch.cuda.current_stream().cuda_stream)
    assert rc == _lib.MXB_ERR_ARG
    assert b"device memory" in lib.mxb_last_error()
    # host W with device pools is refused the same way
    keep2 = []
    ddesc = _device_desc(torch, cds, keep2)
    Wh = np.zeros(cds.n * r)
    rc = lib.mxb_evaluate_noalloc(ctypes.byref(ddesc), Wh.ctypes.data, Y.data_ptr(), r, 0,
                                  torch.cuda.current_stream().cuda_stream)
    assert rc == _lib.MXB_ERR_ARG
    torch.cuda.synchronize()


def test_noalloc_refuses_a_capturing_stream(torch):
    """Each call copies its task lists from temporary host memory, so a capturing stream is
    refused with MXB_ERR_UNSUPPORTED (nothing is enqueued) instead of recording copies that
    would read freed host memory on replay."""
    lib = _lib.load()
    name, cds = next(_cases())
    keep = []
    desc = _device_desc(torch, cds, keep)
    r = 4
    W = torch.zeros(cds.n * r, dtype=torch.float64, device="cuda")
    Y = torch.zeros_like(W)
    side = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(side):
        g.capture_begin()
        try:
            rc = lib.mxb_evaluate_noalloc(ctypes.byref(desc), W.data_ptr(), Y.data_ptr(), r, 0,
                                          side.cuda_stream)
            Y.add_(1.0)  # keeps the captured graph non-empty
        finally:
            g.capture_end()
    assert rc == _lib.MXB_ERR_UNSUPPORTED
    assert b"capturing" in lib.mxb_last_error()
    del g
    torch.cuda.synchronize()
