"""Loader of libmatrox_b200.so and ctypes prototypes of its C-ABI (include/matrox_b200.h).

There is no fallback: if the CUDA library is missing or fails to load, every call raises.
"""
from __future__ import annotations

import ctypes
import os
import re

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libmatrox_b200.so")
HEADER = os.path.join(os.path.dirname(PKG), "include", "matrox_b200.h")

MXB_OK = 0
MXB_ERR_ARG = -1
MXB_ERR_STRUCTURE = -2
MXB_ERR_CUDA = -3
MXB_ERR_NOMEM = -4
MXB_ERR_TIMEOUT = -5
MXB_ERR_UNSUPPORTED = -6
MXB_CACHE_SAMPLED, MXB_CACHE_FULL, MXB_CACHE_OFF = 0, 1, 2
PREC_FP64 = 0
PREC_SPLIT_BF16 = 1
PREC_SPLIT_BF16_FAR6 = 2
PREC_SPLIT_BF16_X6 = 3
FLAG_MIRROR_WORKSPACES = 1
FLAG_OUTPUT_IS_ZERO = 2
DEBUG_STALL_ONE_WAIT = 1
DEBUG_CHAIN_LEVELS = 2
DEBUG_STALL_LEVEL = 4
DEBUG_ONE_LAUNCH = 8
BATCH_LEVEL_LAUNCHES, BATCH_ONE_LAUNCH = 0, 1
TILE_PAIR = 4096
PLAN_ADJOINT = 0x100  # MXB_PLAN_ADJOINT: OR'd into the precision of mxb_plan_create
KERNEL_KINDS = {"gaussian": 0, "imq": 1, "newton": 2}
PHASES = {0: "split_w", 1: "up", 2: "far", 3: "down", 4: "near", 5: "leaf_down", 6: "far_down",
          7: "near_leaf_down", 8: "far_near"}

P = ctypes.c_void_p
I32 = ctypes.c_int32
I64 = ctypes.c_int64
U32 = ctypes.c_uint32
U64 = ctypes.c_uint64


class MxbError(RuntimeError):
    def __init__(self, code: int, where: str, msg: str):
        super().__init__(f"{where} failed with {code}: {msg}")
        self.code = code


class CdsDesc(ctypes.Structure):
    _fields_ = [
        ("nleaf", I32), ("numnodes", I32), ("is_hss", I32),
        ("D", P), ("D_len", U64),
        ("B", P), ("B_len", U64),
        ("VT", P), ("VT_len", U64),
        ("Dptr", P), ("Bptr", P), ("VTptr", P),
        ("lchildren", P), ("rchildren", P), ("lm", P), ("slen", P), ("Ddim", P),
        ("npairx", P), ("npairy", P), ("ncount", I32),
        ("fpairx", P), ("fpairy", P), ("fcount", I32),
    ]


class OpProfile(ctypes.Structure):
    _fields_ = [("phase", I32), ("level", I32), ("width", I32), ("units", I32),
                ("flops", ctypes.c_double), ("issued_flops", ctypes.c_double), ("ms", ctypes.c_float),
                ("pair", I32), ("chained", I32), ("level_ms", ctypes.c_float)]


_REF_ARGS_H2B = [P] * 12 + [I32] + [P] * 9 + [P] * 8  # up to fpairy
_lib = None


def exported_names_from_header(path: str = HEADER):
    """Function names declared with MXB_API in the public header."""
    text = open(path).read()
    return re.findall(r"MXB_API\s+(?:const\s+char\s*\*|int32_t)\s*([A-Za-z_][A-Za-z0-9_]*)\s*\(", text)


def load(path: str = LIB_PATH):
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(
            f"{path} is missing: build it with `python -m matrox_ru_b200.build` (nvcc, sm_100a)")
    lib = ctypes.CDLL(path)
    lib.mxb_last_error.restype = ctypes.c_char_p
    lib.mxb_version.restype = ctypes.c_char_p
    for name in exported_names_from_header():
        f = getattr(lib, name)
        if name not in ("mxb_last_error", "mxb_version"):
            f.restype = I32
    lib.mxb_set_precision.argtypes = [I32]
    lib.mxb_set_flags.argtypes = [U32]
    lib.mxb_cache_set_mode.argtypes = [I32]
    lib.mxb_debug_dataflow_order.argtypes = [I32, P, P, P, P, I32, I32, P, P, P, P, P, P, I64,
                                             ctypes.POINTER(I64)]
    lib.mxb_batch_set_launch_mode.argtypes = [P, I32]
    lib.mxb_plan_create.argtypes = [ctypes.POINTER(CdsDesc), I32, ctypes.POINTER(P)]
    lib.mxb_plan_destroy.argtypes = [P]
    lib.mxb_plan_evaluate.argtypes = [P, P, P, I32, P, P, I32, P]
    lib.mxb_plan_adjoint.argtypes = [P, P, P, I32, P, P, I32, P]
    lib.mxb_plan_set_permutation.argtypes = [P, P]
    lib.mxb_plan_evaluate_ordered.argtypes = [P, P, I64, I64, P, I64, I64, I32, I32, P]
    lib.mxb_plan_adjoint_ordered.argtypes = [P, P, I64, I64, P, I64, I64, I32, I32, P]
    lib.mxb_plan_flops.argtypes = [P, I32, ctypes.POINTER(U64)]
    lib.mxb_plan_info.argtypes = [P, ctypes.POINTER(U64), ctypes.POINTER(I32), ctypes.POINTER(I32)]
    lib.mxb_plan_read_workspaces.argtypes = [P, I32, P, P, P, P]
    lib.mxb_plan_status.argtypes = [P]
    lib.mxb_batch_create.argtypes = [ctypes.POINTER(P), I32, ctypes.POINTER(P)]
    lib.mxb_batch_evaluate.argtypes = [P, ctypes.POINTER(P), ctypes.POINTER(P), ctypes.POINTER(I32), I32, P]
    lib.mxb_batch_status.argtypes = [P]
    lib.mxb_batch_info.argtypes = [P, ctypes.POINTER(I32), ctypes.POINTER(I32), I32, ctypes.POINTER(I32)]
    lib.mxb_batch_destroy.argtypes = [P]
    lib.mxb_plan_profile.argtypes = [P, P, P, I32, P, ctypes.POINTER(OpProfile), I32, ctypes.POINTER(I32)]
    lib.mxb_batch_profile.argtypes = [P, ctypes.POINTER(P), ctypes.POINTER(P), ctypes.POINTER(I32), P,
                                      ctypes.POINTER(OpProfile), I32, ctypes.POINTER(I32)]
    lib.mxb_plan_set_test_hooks.argtypes = [P, I32, I64]
    lib.mxb_permute_rows.argtypes = [P, P, P, I32, I64, P, P, I64, I64, I32, I32, I32, P]
    lib.mxb_transform.argtypes = [P, P, P, I32, P, I64, I64, I32, P]
    lib.mxb_untransform.argtypes = [P, P, P, I32, P, I64, I64, I32, P]
    lib.mxb_evaluate_noalloc.argtypes = [ctypes.POINTER(CdsDesc), P, P, I32, I32, P]
    lib.mxb_batched_id.argtypes = [P, P, P, I32, ctypes.c_double, I32, P, P, P, P]
    lib.mxb_kernel_blocks.argtypes = [P, I64, I32, I32, ctypes.c_double, P, P, I32, P, P, P, I32, P, U64, P]
    lib.mxb_hgemm_set_shape.argtypes = [I32, I32, I32]
    lib.mxb_hgemm_hss_set_shape.argtypes = [I32, I32]
    cb = _REF_ARGS_H2B + [I32, I32, P, P, ctypes.c_int]
    lib.CBHGEMM.argtypes = cb
    lib.lowH2GEMM.argtypes = cb
    lib.blockGEMM.argtypes = _REF_ARGS_H2B + [I32, I32, I32]
    lib.HGEMM.argtypes = _REF_ARGS_H2B + [P, P]
    hss = [P] * 12 + [I32] + [P] * 9
    lib.parHSSGEMM.argtypes = hss + [P, P, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    lib.lowHSSGEMM.argtypes = hss + [P, P, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    lib.seqHSSGEMM.argtypes = hss + [I32, I32, I32]
    lib.HGEMM_HSS.argtypes = hss + [P, P]
    _lib = lib
    return lib


def check(rc: int, where: str) -> None:
    if rc != MXB_OK:
        msg = load().mxb_last_error()
        raise MxbError(rc, where, msg.decode() if msg else "")
