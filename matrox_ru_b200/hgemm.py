"""Host-side mirror of MatRox's evaluator interface over the C-ABI.

* :func:`CBHGEMM`, :func:`HGEMM`, :func:`parHSSGEMM` ... call the drop-ins with the
  reference's argument lists, built from a :class:`~matrox_ru_b200.structure.CDS` the way
  ``matroxTest-V1/main.cpp:97-107`` and ``codeTest/main.cpp:111-171`` build them.
* :class:`Plan` wraps the device-pointer plan API for torch tensors.
* :class:`Evaluator` adds the permutation between the caller's point order and the
  leaf-blocked tree order, and the adjoint.
"""
from __future__ import annotations

import ctypes
from typing import Optional

import numpy as np

from . import _lib
from ._lib import P, I32, check

PRECISIONS = {"fp64": _lib.PREC_FP64, "split_bf16": _lib.PREC_SPLIT_BF16,
              "split_bf16_far6": _lib.PREC_SPLIT_BF16_FAR6, "split_bf16_x6": _lib.PREC_SPLIT_BF16_X6}


def _np(a, dt):
    a = np.ascontiguousarray(a, dtype=dt)
    if a.size == 0:
        a = np.zeros(1, dt)
    return a


class _Args:
    """Keeps the numpy arrays of one drop-in call alive and hands out their pointers."""

    def __init__(self):
        self.keep = []

    def __call__(self, a, dt=np.int32):
        a = _np(a, dt)
        self.keep.append(a)
        return a.ctypes.data_as(P)


def set_precision(mode: str) -> None:
    check(_lib.load().mxb_set_precision(PRECISIONS[mode]), "mxb_set_precision")


def set_flags(flags: int) -> None:
    check(_lib.load().mxb_set_flags(flags), "mxb_set_flags")


def cache_invalidate() -> None:
    check(_lib.load().mxb_cache_invalidate(), "mxb_cache_invalidate")


CACHE_MODES = {"sampled": _lib.MXB_CACHE_SAMPLED, "full": _lib.MXB_CACHE_FULL, "off": _lib.MXB_CACHE_OFF}


def cache_set_mode(mode: str) -> None:
    """How the drop-ins recognise an uploaded CDS: "sampled" (default), "full" or "off"."""
    check(_lib.load().mxb_cache_set_mode(CACHE_MODES[mode]), "mxb_cache_set_mode")


def _ref_args(cds, TW, apres, nrhs, wskel, uskel, idx):
    a = _Args()
    wptr, uptr, wsko, usko, _ = cds.offsets(nrhs)
    args = [a(cds.D, np.float64), a(cds.B, np.float64), a(cds.VT, np.float64), a(cds.Dptr, np.uint64),
            a(cds.Bptr, np.uint64), a(cds.VTptr), a(cds.lchildren), a(cds.rchildren), a(cds.levelset),
            a(idx), TW.ctypes.data_as(P), apres.ctypes.data_as(P), I32(nrhs), a(cds.Ddim), a(wptr),
            a(uptr), wskel.ctypes.data_as(P), a(wsko), uskel.ctypes.data_as(P), a(usko), a(cds.lm),
            a(cds.slen)]
    return a, args


def _work(cds, nrhs, wskel, uskel):
    n = max(int(cds.slen.astype(np.int64).sum()) * nrhs, 1)
    if wskel is None:
        wskel = np.zeros(n)
    if uskel is None:
        uskel = np.zeros(n)
    return wskel, uskel


def CBHGEMM(cds, TW: np.ndarray, apres: np.ndarray, nrhs: int, wskel=None, uskel=None,
            variant: str = "CBHGEMM") -> int:
    """Drop-in H2-b evaluation on host arrays (``codeGen/H2GEMM.h:380``):
    apres += K~ TW, both leaf-blocked FP64 arrays of N * nrhs elements."""
    if cds.is_hss:
        raise ValueError("CBHGEMM takes an H2-b CDS; use parHSSGEMM for HSS")
    lib = _lib.load()
    wskel, uskel = _work(cds, nrhs, wskel, uskel)
    idx = cds.idx if variant == "blockGEMM" else cds.cidx
    a, args = _ref_args(cds, TW, apres, nrhs, wskel, uskel, idx)
    args += [a(cds.nblockset), a(cds.nblocks), a(cds.npairx), a(cds.npairy), a(cds.fblockset),
             a(cds.fblocks), a(cds.fpairx), a(cds.fpairy)]
    if variant in ("CBHGEMM", "lowH2GEMM"):
        args += [I32(cds.nrow), I32(cds.frow), a(cds.wpart), a(cds.clevelset), ctypes.c_int(cds.cdepth)]
        rc = getattr(lib, variant)(*args)
    elif variant == "blockGEMM":
        args += [I32(cds.nrow), I32(cds.frow), I32(cds.depth)]
        rc = lib.blockGEMM(*args)
    elif variant == "HGEMM":
        check(lib.mxb_hgemm_set_shape(cds.nrow, cds.frow, cds.cdepth), "mxb_hgemm_set_shape")
        args += [a(cds.wpart), a(cds.clevelset)]
        rc = lib.HGEMM(*args)
    else:
        raise ValueError(variant)
    check(rc, variant)
    return rc


def parHSSGEMM(cds, TW: np.ndarray, apres: np.ndarray, nrhs: int, wskel=None, uskel=None,
               variant: str = "parHSSGEMM") -> int:
    """Drop-in HSS evaluation on host arrays (``codeGen/HSSGEMM.h:131``):
    apres = K~ TW (the HSS near pass overwrites)."""
    if not cds.is_hss:
        raise ValueError("parHSSGEMM takes an HSS CDS")
    lib = _lib.load()
    wskel, uskel = _work(cds, nrhs, wskel, uskel)
    idx = cds.idx if variant == "seqHSSGEMM" else cds.cidx
    a, args = _ref_args(cds, TW, apres, nrhs, wskel, uskel, idx)
    if variant in ("parHSSGEMM", "lowHSSGEMM"):
        args += [a(cds.wpart), a(cds.clevelset), ctypes.c_int(cds.nleaf), ctypes.c_int(cds.numnodes - 1),
                 ctypes.c_int(cds.cdepth)]
        rc = getattr(lib, variant)(*args)
    elif variant == "seqHSSGEMM":
        args += [I32(cds.nleaf), I32(cds.numnodes - 1), I32(cds.depth)]
        rc = lib.seqHSSGEMM(*args)
    elif variant == "HGEMM_HSS":
        check(lib.mxb_hgemm_hss_set_shape(cds.nleaf, cds.cdepth), "mxb_hgemm_hss_set_shape")
        args += [a(cds.wpart), a(cds.clevelset)]
        rc = lib.HGEMM_HSS(*args)
    else:
        raise ValueError(variant)
    check(rc, variant)
    return rc


def evaluate_host(cds, TW: np.ndarray, nrhs: int, apres: Optional[np.ndarray] = None) -> np.ndarray:
    """Reference-style host call of whichever drop-in matches the CDS (apres zeroed if None)."""
    TW = np.ascontiguousarray(TW, dtype=np.float64)
    if apres is None:
        apres = np.zeros_like(TW)
    (parHSSGEMM if cds.is_hss else CBHGEMM)(cds, TW, apres, nrhs)
    return apres


def transform(cds, W: np.ndarray, nrhs: int) -> np.ndarray:
    """``transform`` (``hcds.h:766``) on the GPU: W (N x nrhs, column-major) -> TW."""
    lib = _lib.load()
    W = np.asfortranarray(W, dtype=np.float64)
    wptr = cds.offsets(nrhs)[0]
    TW = np.zeros(cds.n * nrhs)
    a = _Args()
    check(lib.mxb_transform(a(cds.perm), a(cds.leaf_lids_offset), a(wptr), cds.nleaf, W.ctypes.data_as(P),
                            cds.n, cds.n, nrhs, TW.ctypes.data_as(P)), "mxb_transform")
    return TW


def untransform(cds, TY: np.ndarray, nrhs: int) -> np.ndarray:
    lib = _lib.load()
    uptr = cds.offsets(nrhs)[1]
    Y = np.zeros((cds.n, nrhs), order="F")
    a = _Args()
    check(lib.mxb_untransform(a(cds.perm), a(cds.leaf_lids_offset), a(uptr), cds.nleaf,
                              a(TY, np.float64), cds.n, cds.n, nrhs, Y.ctypes.data_as(P)), "mxb_untransform")
    return Y


# -----------------------------------------------------------------------------------------
# device plans (torch tensors)
# -----------------------------------------------------------------------------------------

def _torch():
    import torch
    return torch


def _stream_ptr(stream) -> int:
    torch = _torch()
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream


def cds_desc(cds, keep: list) -> _lib.CdsDesc:
    def k(a, dt=np.int32):
        a = _np(a, dt)
        keep.append(a)
        return a.ctypes.data

    d = _lib.CdsDesc()
    d.nleaf, d.numnodes, d.is_hss = cds.nleaf, cds.numnodes, int(cds.is_hss)
    d.D, d.D_len = k(cds.D, np.float64), cds.D.size
    d.B, d.B_len = k(cds.B, np.float64), cds.B.size
    d.VT, d.VT_len = k(cds.VT, np.float64), cds.VT.size
    d.Dptr, d.Bptr, d.VTptr = k(cds.Dptr, np.uint64), k(cds.Bptr, np.uint64), k(cds.VTptr)
    d.lchildren, d.rchildren, d.lm, d.slen, d.Ddim = (k(cds.lchildren), k(cds.rchildren), k(cds.lm),
                                                      k(cds.slen), k(cds.Ddim))
    d.npairx, d.npairy, d.ncount = k(cds.npairx), k(cds.npairy), cds.ncount
    d.fpairx, d.fpairy, d.fcount = k(cds.fpairx), k(cds.fpairy), cds.fcount
    return d


def _profile_records(recs, n):
    return [{"phase": _lib.PHASES.get(r.phase, str(r.phase)), "level": r.level, "width": r.width, "units": r.units,
             "pair": bool(r.pair), "chained": bool(r.chained), "flops": r.flops, "issued_flops": r.issued_flops,
             "ms": r.ms, "level_ms": r.level_ms} for r in recs[:min(n, len(recs))]]


def kernel_blocks(cds, X, kernel, stream=None):
    """The CDS's near blocks D and far couplings B computed on the GPU from the points
    (``mxb_kernel_blocks``; the reference computes them on the host with ``Fsubmatrix``,
    ``matroxTest-V1/compression.h:256-360``).  X: (N, d) float64 points, host or CUDA;
    kernel: a :class:`~matrox_ru_b200.structure.KernelSpec`.  Returns CUDA tensors (D, B) in the
    layout of ``cds.D`` / ``cds.B`` (offsets ``cds.Dptr`` / ``cds.Bptr``)."""
    torch = _torch()
    dX = torch.as_tensor(np.ascontiguousarray(X, dtype=np.float64)).to("cuda")
    n, d = dX.shape
    # index sets: the points of every leaf (tree order), then the skeleton points of every node
    leaf_sets = [cds.perm[int(cds.leaf_lids_offset[i]):int(cds.leaf_lids_offset[i + 1])] for i in range(cds.nleaf)]
    skel_sets = [np.asarray(s if s is not None else [], dtype=np.int64) for s in cds.skels]
    sets = leaf_sets + skel_sets
    set_ofs = np.concatenate([[0], np.cumsum([len(s) for s in sets])]).astype(np.int64)
    set_idx = np.concatenate(sets).astype(np.int32) if len(set_ofs) > 1 and set_ofs[-1] else np.zeros(1, np.int32)
    nl = cds.nleaf
    # the near pair list holds leaf indices; far pairs hold node indices
    out = []
    for rows, cols, ofs, length in ((np.asarray(cds.npairx), np.asarray(cds.npairy), cds.Dptr, cds.D.size),
                                    (np.asarray(cds.fpairx) + nl, np.asarray(cds.fpairy) + nl, cds.Bptr, cds.B.size)):
        dst = torch.empty(max(int(length), 1), dtype=torch.float64, device=dX.device)
        a = _Args()
        check(_lib.load().mxb_kernel_blocks(dX.data_ptr(), n, d, _lib.KERNEL_KINDS[kernel.kind], float(kernel.h),
                                            a(set_ofs, np.int64), a(set_idx), len(sets), a(rows), a(cols),
                                            a(ofs, np.uint64), len(rows), dst.data_ptr(), int(length),
                                            _stream_ptr(stream)), "mxb_kernel_blocks")
        out.append(dst)
    return out[0], out[1]


def kernel_matrices(dX, kernel, row_sets, col_sets, stream=None):
    """Kernel blocks K(X[rows_b], X[cols_b]) for every pair of index sets, computed on the GPU
    (``mxb_kernel_blocks``) and packed back to back, each column-major.  dX: (N, d) float64
    CUDA tensor.  Returns (pool, offsets)."""
    torch = _torch()
    n, d = dX.shape
    sets = [np.asarray(x, dtype=np.int64) for x in row_sets] + [np.asarray(x, dtype=np.int64) for x in col_sets]
    nb = len(row_sets)
    set_ofs = np.concatenate([[0], np.cumsum([len(x) for x in sets])]).astype(np.int64)
    set_idx = np.concatenate(sets).astype(np.int32) if set_ofs[-1] else np.zeros(1, np.int32)
    sizes = np.array([len(r) * len(c) for r, c in zip(row_sets, col_sets)], np.int64)
    ofs = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.uint64)
    total = int(sizes.sum())
    dst = torch.empty(max(total, 1), dtype=torch.float64, device=dX.device)
    a = _Args()
    check(_lib.load().mxb_kernel_blocks(dX.data_ptr(), n, d, _lib.KERNEL_KINDS[kernel.kind], float(kernel.h),
                                        a(set_ofs, np.int64), a(set_idx), len(sets),
                                        a(np.arange(nb, dtype=np.int32)), a(np.arange(nb, 2 * nb, dtype=np.int32)),
                                        a(ofs, np.uint64), nb, dst.data_ptr(), total, _stream_ptr(stream)),
          "mxb_kernel_blocks")
    return dst, ofs


def batched_id(pool, shapes, tol: float, max_rank: int, stream=None):
    """Column IDs of the packed column-major matrices in ``pool`` (a float64 CUDA tensor,
    overwritten), ``shapes`` = [(nrows, ncols), ...], on the GPU (``mxb_batched_id``).  Returns a
    list of (skeleton column positions, P) as numpy arrays, like
    :func:`matrox_ru_b200.structure.interpolative_decomposition`."""
    torch = _torch()
    if not shapes:
        return []
    nr = np.array([r for r, _ in shapes], np.int32)
    nc = np.array([c for _, c in shapes], np.int32)
    if not (pool.is_cuda and pool.dtype == torch.float64 and pool.is_contiguous()):
        raise TypeError("pool must be a contiguous float64 CUDA tensor")
    if pool.numel() < int((nr.astype(np.int64) * nc).sum()):
        raise ValueError("pool smaller than the matrices it should hold")
    pmax = np.minimum(max_rank, nc).astype(np.int64)
    dRank = torch.empty(len(shapes), dtype=torch.int32, device=pool.device)
    dPiv = torch.empty(int(nc.sum()), dtype=torch.int32, device=pool.device)
    dP = torch.empty(max(int((pmax * nc).sum()), 1), dtype=torch.float64, device=pool.device)
    check(_lib.load().mxb_batched_id(pool.data_ptr(), nr.ctypes.data, nc.ctypes.data, len(shapes), float(tol),
                                     int(max_rank), dRank.data_ptr(), dPiv.data_ptr(), dP.data_ptr(),
                                     _stream_ptr(stream)), "mxb_batched_id")
    ranks = dRank.cpu().numpy()
    piv = dPiv.cpu().numpy()
    Pall = dP.cpu().numpy()
    out, q, p = [], 0, 0
    for b in range(len(shapes)):
        s, c = int(ranks[b]), int(nc[b])
        out.append((piv[q:q + s].astype(np.int64), Pall[p:p + s * c].reshape(s, c, order="F").copy()))
        q += c
        p += int(pmax[b]) * c
    return out


class Plan:
    """Device-resident CDS and task lists (``mxb_plan_*``).  ``pools`` optionally gives the
    numeric pools (D, B, VT) as CUDA tensors (e.g. from :func:`kernel_blocks`) instead of the
    CDS's host arrays.  ``adjoint``: a split-BF16 plan also tiles the transposed near blocks and
    far couplings, so :meth:`adjoint` runs on the tensor cores (``MXB_PLAN_ADJOINT``); FP64 plans
    always have the adjoint."""

    def __init__(self, cds, precision: str = "fp64", pools=None, adjoint: bool = False):
        torch = _torch()
        if not torch.cuda.is_available():
            raise RuntimeError("matrox_ru_b200.Plan needs a CUDA device")
        lib = _lib.load()
        keep: list = []
        desc = cds_desc(cds, keep)
        if pools is not None:
            for name, t in zip(("D", "B", "VT"), pools):
                if t is None:
                    continue
                if not (t.is_cuda and t.dtype == torch.float64 and t.is_contiguous()):
                    raise TypeError("device pools must be contiguous float64 CUDA tensors")
                if t.numel() < getattr(cds, name).size:
                    raise ValueError(f"device pool {name} is smaller than the CDS's")
                keep.append(t)
                setattr(desc, name, t.data_ptr())
            torch.cuda.synchronize()  # the pools were written on torch's stream
        h = P()
        code = PRECISIONS[precision] | (_lib.PLAN_ADJOINT if adjoint and precision != "fp64" else 0)
        check(lib.mxb_plan_create(ctypes.byref(desc), code, ctypes.byref(h)), "mxb_plan_create")
        self._h = h
        self.cds = cds
        self.precision = precision
        self.n = cds.n
        self.device = torch.cuda.current_device()

    def close(self):
        if getattr(self, "_h", None):
            _lib.load().mxb_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def flops(self, nrhs: int) -> int:
        f = _lib.U64()
        check(_lib.load().mxb_plan_flops(self._h, nrhs, ctypes.byref(f)), "mxb_plan_flops")
        return int(f.value)

    def info(self):
        b, l, p = _lib.U64(), I32(), I32()
        check(_lib.load().mxb_plan_info(self._h, ctypes.byref(b), ctypes.byref(l), ctypes.byref(p)), "mxb_plan_info")
        return {"device_bytes": int(b.value), "launches": int(l.value), "precision": int(p.value)}

    def set_test_hooks(self, flags: int, wait_cycles: int = 0) -> None:
        """Failure-detection test hook (see mxb_plan_set_test_hooks)."""
        check(_lib.load().mxb_plan_set_test_hooks(self._h, flags, wait_cycles), "mxb_plan_set_test_hooks")

    def status(self) -> None:
        """Synchronise and raise if a kernel of an earlier evaluation reported a failure."""
        check(_lib.load().mxb_plan_status(self._h), "mxb_plan_status")

    def _check_operand(self, t, nrhs):
        torch = _torch()
        if not (t.is_cuda and t.dtype == torch.float64 and t.is_contiguous()):
            raise TypeError("operands must be contiguous float64 CUDA tensors")
        if t.numel() < self.n * nrhs:
            raise ValueError("operand smaller than N * nrhs")

    def evaluate(self, TW, nrhs: int, out=None, accumulate: bool = False, stream=None):
        """out (+)= K~ TW on packed leaf-blocked float64 CUDA tensors (N * nrhs)."""
        torch = _torch()
        self._check_operand(TW, nrhs)
        if out is None:
            out = torch.zeros(self.n * nrhs, dtype=torch.float64, device=TW.device)
            accumulate = False
        self._check_operand(out, nrhs)
        check(_lib.load().mxb_plan_evaluate(self._h, TW.data_ptr(), out.data_ptr(), nrhs, None, None,
                                            int(accumulate), _stream_ptr(stream)), "mxb_plan_evaluate")
        return out

    def profile(self, TW, nrhs: int, out=None, stream=None):
        """out = K~ TW, then the device time and flops of every launch of one evaluation
        (``mxb_plan_profile``): a list of dicts in launch order."""
        torch = _torch()
        self._check_operand(TW, nrhs)
        if out is None:
            out = torch.zeros(self.n * nrhs, dtype=torch.float64, device=TW.device)
        self._check_operand(out, nrhs)
        recs = (_lib.OpProfile * 4096)()
        n = I32()
        check(_lib.load().mxb_plan_profile(self._h, TW.data_ptr(), out.data_ptr(), nrhs, _stream_ptr(stream),
                                           recs, 4096, ctypes.byref(n)), "mxb_plan_profile")
        return _profile_records(recs, n.value)

    def set_permutation(self, perm) -> None:
        """Register the caller's point order: perm[t] is the row of W / Y that holds tree
        position t (``CDS.perm``, the reference's ``lids``)."""
        perm = np.ascontiguousarray(perm, dtype=np.int32)
        if perm.shape != (self.n,):
            raise ValueError("perm must have one entry per point")
        check(_lib.load().mxb_plan_set_permutation(self._h, perm.ctypes.data), "mxb_plan_set_permutation")

    def _ordered(self, fn, name, W, out, accumulate, stream):
        torch = _torch()
        if not (W.is_cuda and W.dtype == torch.float64 and W.dim() == 2 and W.shape[0] == self.n):
            raise TypeError("operands must be (N, r) float64 CUDA tensors")
        r = W.shape[1]
        if out is None:
            out = torch.empty((self.n, r), dtype=torch.float64, device=W.device)
            accumulate = False
        if not (out.is_cuda and out.dtype == torch.float64 and tuple(out.shape) == (self.n, r)):
            raise TypeError("out must be an (N, r) float64 CUDA tensor")
        check(fn(self._h, W.data_ptr(), W.stride(0), W.stride(1), out.data_ptr(), out.stride(0), out.stride(1), r,
                 int(accumulate), _stream_ptr(stream)), name)
        return out

    def evaluate_ordered(self, W, out=None, accumulate: bool = False, stream=None):
        """out (+)= K~ W with W, out as (N, r) float64 CUDA tensors in the caller's point
        order (any non-overlapping strides).  Split-BF16 plans gather and scatter the rows
        inside their own launches; ``set_permutation`` must have been called."""
        return self._ordered(_lib.load().mxb_plan_evaluate_ordered, "mxb_plan_evaluate_ordered", W, out,
                             accumulate, stream)

    def adjoint_ordered(self, G, out=None, accumulate: bool = False, stream=None):
        """out (+)= K~^T G in the caller's point order (FP64 plans, split-BF16 plans with the
        adjoint)."""
        return self._ordered(_lib.load().mxb_plan_adjoint_ordered, "mxb_plan_adjoint_ordered", G, out,
                             accumulate, stream)

    def adjoint(self, TG, nrhs: int, out=None, accumulate: bool = False, stream=None):
        """out (+)= K~^T TG (packed leaf-blocked float64 CUDA tensors)."""
        torch = _torch()
        self._check_operand(TG, nrhs)
        if out is None:
            out = torch.zeros(self.n * nrhs, dtype=torch.float64, device=TG.device)
            accumulate = False
        self._check_operand(out, nrhs)
        check(_lib.load().mxb_plan_adjoint(self._h, TG.data_ptr(), out.data_ptr(), nrhs, None, None,
                                           int(accumulate), _stream_ptr(stream)), "mxb_plan_adjoint")
        return out


class Batch:
    """Several split-BF16 plans evaluated by one merged, graph-captured launch sequence
    (``mxb_batch_*``); the column-tile widths are tuned by measurement on first use."""

    def __init__(self, plans):
        if not plans:
            raise ValueError("empty batch")
        self.plans = list(plans)  # the plans must outlive the batch
        arr = (P * len(self.plans))(*[p._h for p in self.plans])
        h = P()
        check(_lib.load().mxb_batch_create(arr, len(self.plans), ctypes.byref(h)), "mxb_batch_create")
        self._h = h

    def set_one_launch(self, on: bool = True) -> None:
        """Evaluate the whole batch as one launch with device-side level barriers
        (MXB_BATCH_ONE_LAUNCH), or as a sequence of level launches (the default)."""
        mode = _lib.BATCH_ONE_LAUNCH if on else _lib.BATCH_LEVEL_LAUNCHES
        check(_lib.load().mxb_batch_set_launch_mode(self._h, mode), "mxb_batch_set_launch_mode")

    def close(self):
        if getattr(self, "_h", None):
            _lib.load().mxb_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def evaluate(self, TWs, nrhs, outs=None, accumulate=False, stream=None):
        """outs[i] (+)= K~_i TWs[i] for every plan i (packed leaf-blocked float64 CUDA tensors)."""
        torch = _torch()
        n = len(self.plans)
        if len(TWs) != n or len(nrhs) != n:
            raise ValueError("one operand and one nrhs per plan")
        if outs is None:
            outs = [torch.zeros(p.n * r, dtype=torch.float64, device=t.device)
                    for p, r, t in zip(self.plans, nrhs, TWs)]
            accumulate = False
        for p, r, t, o in zip(self.plans, nrhs, TWs, outs):
            p._check_operand(t, r)
            p._check_operand(o, r)
        W = (P * n)(*[t.data_ptr() for t in TWs])
        Y = (P * n)(*[o.data_ptr() for o in outs])
        R = (I32 * n)(*[int(r) for r in nrhs])
        check(_lib.load().mxb_batch_evaluate(self._h, W, Y, R, int(accumulate), _stream_ptr(stream)),
              "mxb_batch_evaluate")
        return outs

    def status(self) -> None:
        check(_lib.load().mxb_batch_status(self._h), "mxb_batch_status")

    def profile(self, TWs, nrhs, outs, stream=None):
        """outs[i] = K~_i TWs[i], then the device time and flops of every merged launch."""
        n = len(self.plans)
        W = (P * n)(*[t.data_ptr() for t in TWs])
        Y = (P * n)(*[o.data_ptr() for o in outs])
        R = (I32 * n)(*[int(r) for r in nrhs])
        recs = (_lib.OpProfile * 4096)()
        cnt = I32()
        check(_lib.load().mxb_batch_profile(self._h, W, Y, R, _stream_ptr(stream), recs, 4096, ctypes.byref(cnt)),
              "mxb_batch_profile")
        return _profile_records(recs, cnt.value)

    def info(self):
        l, nw = I32(), I32()
        widths = (I32 * 256)()
        check(_lib.load().mxb_batch_info(self._h, ctypes.byref(l), widths, 256, ctypes.byref(nw)), "mxb_batch_info")
        codes = [int(widths[i]) for i in range(nw.value)]
        return {"launches": int(l.value), "widths": [c & (_lib.TILE_PAIR - 1) for c in codes],
                "pairs": [bool(c & _lib.TILE_PAIR) for c in codes]}


class Evaluator:
    """Y = K~ W with W, Y as (N, r) float64 CUDA tensors in the caller's point order."""

    def __init__(self, cds, precision: str = "fp64", plan: Optional[Plan] = None):
        torch = _torch()
        # a split-BF16 evaluator carries the tensor-core adjoint too (its backward pass)
        self.plan = plan if plan is not None else Plan(cds, precision, adjoint=True)
        self.plan.set_permutation(cds.perm)
        self.cds = cds
        dev = torch.device("cuda", self.plan.device)
        self.perm = torch.as_tensor(cds.perm.astype(np.int32), device=dev)
        self.leafofs = torch.as_tensor(cds.leaf_lids_offset.astype(np.int32), device=dev)
        self._blockofs = {}

    def blockofs(self, nrhs: int):
        if nrhs not in self._blockofs:
            torch = _torch()
            offs = (self.cds.leaf_lids_offset[:-1].astype(np.int64) * nrhs)
            if offs.size and offs[-1] > np.iinfo(np.int32).max:
                raise ValueError("leaf offsets overflow int32")
            self._blockofs[nrhs] = torch.as_tensor(offs.astype(np.int32), device=self.perm.device)
        return self._blockofs[nrhs]

    def to_tree(self, W, stream=None):
        torch = _torch()
        n, r = W.shape
        TW = torch.empty(n * r, dtype=torch.float64, device=W.device)
        check(_lib.load().mxb_permute_rows(self.perm.data_ptr(), self.leafofs.data_ptr(),
                                           self.blockofs(r).data_ptr(), self.cds.nleaf, n, W.data_ptr(),
                                           TW.data_ptr(), W.stride(0), W.stride(1), r, 0, 0,
                                           _stream_ptr(stream)), "mxb_permute_rows")
        return TW

    def from_tree(self, TY, r, out=None, accumulate=False, stream=None):
        torch = _torch()
        n = self.cds.n
        if out is None:
            out = torch.empty((n, r), dtype=torch.float64, device=TY.device)
            accumulate = False
        check(_lib.load().mxb_permute_rows(self.perm.data_ptr(), self.leafofs.data_ptr(),
                                           self.blockofs(r).data_ptr(), self.cds.nleaf, n, TY.data_ptr(),
                                           out.data_ptr(), out.stride(0), out.stride(1), r, 1, int(accumulate),
                                           _stream_ptr(stream)), "mxb_permute_rows")
        return out

    def __call__(self, W, stream=None):
        torch = _torch()
        if W.dtype != torch.float64 or not W.is_cuda or W.dim() != 2 or W.shape[0] != self.cds.n:
            raise TypeError("W must be an (N, r) float64 CUDA tensor")
        return self.plan.evaluate_ordered(W, stream=stream)

    def adjoint(self, G, stream=None):
        return self.plan.adjoint_ordered(G, stream=stream)


def kernel_matvec(evaluator: Evaluator, W):
    """Differentiable Y = K~ W (gradient by the transposed traversal)."""
    from .autograd import KernelMatVec
    return KernelMatVec.apply(W, evaluator)
