"""ORACLE -- test infrastructure only.

ctypes front end of the two CPU checkers built by ``oracle/Makefile``:

* ``liboracle_hgemm.so``: this repository's plain-C FP64 restatement of the reference
  evaluator (``hgemm_oracle.c``; follows ``symGen/HGEMM_gen.h:120-238``,
  ``codeGen/H2GEMM.h:380-504`` and ``codeGen/HSSGEMM.h:131-243``);
* ``_ref/libmatrox_ref.so``: the reference's own ``CBHGEMM`` / ``blockGEMM`` /
  ``parHSSGEMM`` / ``seqHSSGEMM`` compiled from its sources (present only where the
  reference tree was available at build time; the library travels with the repository
  snapshot).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import this.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "liboracle_hgemm.so")
REF_SO = os.path.join(HERE, "_ref", "libmatrox_ref.so")

_P = ctypes.c_void_p
_I = ctypes.c_int32


def build(quiet: bool = True) -> None:
    """Run the oracle Makefile (restatement always; reference when its sources exist)."""
    out = subprocess.run(["make", "-C", HERE], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)
    if not quiet:
        print(out.stdout)


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(_P)


_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build()
        _lib = ctypes.CDLL(ORACLE_SO)
        for name in ("oracle_h2b", "oracle_hss", "oracle_adjoint"):
            getattr(_lib, name).restype = _I
    return _lib


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref():
    global _ref
    if _ref is None:
        if not ref_available():
            raise FileNotFoundError("reference evaluator library not built (oracle/_ref)")
        _ref = ctypes.CDLL(REF_SO)
        for name in ("ref_CBHGEMM", "ref_blockGEMM", "ref_parHSSGEMM", "ref_seqHSSGEMM"):
            getattr(_ref, name).restype = _I
        _ref.ref_get_omp_threads.restype = ctypes.c_int
        _ref.ref_set_blas_threads(1)
    return _ref


def ref_decomposition(A: np.ndarray, tol: float):
    """The reference's own column ID, ``decomposition`` (matroxTest-V1/compression.h:446-523:
    dgeqp3, the rank rule with its maximum rank of 256 as written there, dtrsm), of A
    (nrows > ncols).  Returns (skeleton columns, P) like
    ``structure.interpolative_decomposition``."""
    lib = ref()
    a = np.array(A, dtype=np.float64, order="F", copy=True)
    nr, nc = a.shape
    sk = ctypes.POINTER(ctypes.c_int)()
    pr = ctypes.POINTER(ctypes.c_double)()
    jp = ctypes.POINTER(ctypes.c_int)()
    lib.ref_decomposition.restype = ctypes.c_int
    lib.ref_decomposition.argtypes = [_P, ctypes.c_int, ctypes.c_int, ctypes.c_double, _P, _P, _P]
    s = lib.ref_decomposition(a.ctypes.data_as(_P), nr, nc, tol, ctypes.byref(sk), ctypes.byref(pr),
                              ctypes.byref(jp))
    skels = np.ctypeslib.as_array(sk, shape=(s,)).astype(np.int64).copy()
    P = np.ctypeslib.as_array(pr, shape=(s * nc,)).reshape(s, nc, order="F").copy()
    lib.ref_id_free.argtypes = [_P]
    for q in (sk, pr, jp):
        lib.ref_id_free(ctypes.cast(q, _P))
    return skels, P


class Workspace:
    """Host arrays of one evaluation in the reference's layout for a given nrhs."""

    def __init__(self, cds, nrhs: int):
        self.cds = cds
        self.nrhs = nrhs
        self.wptr, self.uptr, self.wsko, self.usko, self.nskel = cds.offsets(nrhs)
        self.wskel = np.zeros(max(self.nskel, 1))
        self.uskel = np.zeros(max(self.nskel, 1))

    def reset(self):
        self.wskel[:] = 0
        self.uskel[:] = 0


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


def _common(cds, ws, TW, Y):
    i32 = np.int32
    return [_ptr(_c(cds.D, np.float64)), _ptr(_c(cds.B if cds.B.size else np.zeros(1), np.float64)),
            _ptr(_c(cds.VT if cds.VT.size else np.zeros(1), np.float64)),
            _ptr(_c(cds.Dptr, np.uint64)), _ptr(_c(cds.Bptr if cds.Bptr.size else np.zeros(1, np.uint64), np.uint64)),
            _ptr(_c(cds.VTptr, i32)), _ptr(_c(cds.lchildren, i32)), _ptr(_c(cds.rchildren, i32)),
            _ptr(_c(cds.levelset, i32))]


def eval_h2b(cds, TW: np.ndarray, nrhs: int, Y: Optional[np.ndarray] = None,
             use_reference: bool = False, ws: Optional[Workspace] = None) -> np.ndarray:
    """Y += K~ TW (tree order, leaf-blocked, FP64) with the restatement or the reference."""
    ws = ws or Workspace(cds, nrhs)
    ws.reset()
    TW = _c(TW, np.float64)
    if Y is None:
        Y = np.zeros_like(TW)
    keep = []

    def k(a, dt=np.int32):
        a = _c(a if np.asarray(a).size else np.zeros(1, dt), dt)
        keep.append(a)
        return a.ctypes.data_as(_P)

    args = [k(cds.D, np.float64), k(cds.B, np.float64), k(cds.VT, np.float64),
            k(cds.Dptr, np.uint64), k(cds.Bptr, np.uint64), k(cds.VTptr), k(cds.lchildren),
            k(cds.rchildren), k(cds.levelset), k(cds.cidx), TW.ctypes.data_as(_P),
            Y.ctypes.data_as(_P), _I(nrhs), k(cds.Ddim), k(ws.wptr), k(ws.uptr),
            ws.wskel.ctypes.data_as(_P), k(ws.wsko), ws.uskel.ctypes.data_as(_P), k(ws.usko),
            k(cds.lm), k(cds.slen)]
    if cds.is_hss:
        args += [k(cds.wpart), k(cds.clevelset), _I(cds.nleaf), _I(cds.numnodes - 1), _I(cds.cdepth)]
        fn = ref().ref_parHSSGEMM if use_reference else lib().oracle_hss
    else:
        args += [k(cds.nblockset), k(cds.nblocks), k(cds.npairx), k(cds.npairy), k(cds.fblockset),
                 k(cds.fblocks), k(cds.fpairx), k(cds.fpairy), _I(cds.nrow), _I(cds.frow),
                 k(cds.wpart), k(cds.clevelset), _I(cds.cdepth)]
        fn = ref().ref_CBHGEMM if use_reference else lib().oracle_h2b
    rc = fn(*args)
    if rc != 0:
        raise RuntimeError(f"oracle evaluation returned {rc}")
    return Y


def adjoint(cds, G: np.ndarray, nrhs: int, GW: Optional[np.ndarray] = None) -> np.ndarray:
    """GW += K~^T G (tree order) by the transposed traversal."""
    ws = Workspace(cds, nrhs)
    G = _c(G, np.float64)
    if GW is None:
        GW = np.zeros_like(G)
    keep = []

    def k(a, dt=np.int32):
        a = _c(a if np.asarray(a).size else np.zeros(1, dt), dt)
        keep.append(a)
        return a.ctypes.data_as(_P)

    rc = lib().oracle_adjoint(
        k(cds.D, np.float64), k(cds.B, np.float64), k(cds.VT, np.float64), k(cds.Dptr, np.uint64),
        k(cds.Bptr, np.uint64), k(cds.VTptr), k(cds.lchildren), k(cds.rchildren), k(cds.cidx),
        G.ctypes.data_as(_P), GW.ctypes.data_as(_P), _I(nrhs), k(cds.Ddim), k(ws.wptr), k(ws.uptr),
        ws.wskel.ctypes.data_as(_P), k(ws.wsko), ws.uskel.ctypes.data_as(_P), k(ws.usko), k(cds.lm),
        k(cds.slen), k(cds.npairx), k(cds.npairy), _I(cds.ncount), k(cds.fpairx), k(cds.fpairy),
        _I(cds.fcount), k(cds.wpart), k(cds.clevelset), _I(cds.cdepth))
    if rc != 0:
        raise RuntimeError(f"oracle adjoint returned {rc}")
    return GW
