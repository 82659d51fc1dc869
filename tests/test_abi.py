"""CPU: the C-ABI library builds for sm_100a, loads, and exports every symbol the header
declares (no compute calls: there is no GPU here)."""
import ctypes
import os
import subprocess

import pytest

from matrox_ru_b200 import _lib, build


@pytest.fixture(scope="module")
def lib_path():
    return build.build()


def test_exports_match_header(lib_path):
    names = _lib.exported_names_from_header()
    assert len(names) >= 20
    out = subprocess.run(["nm", "-D", "--defined-only", lib_path], capture_output=True, text=True).stdout
    exported = {l.split()[-1] for l in out.splitlines() if " T " in l}
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    # nothing but the header's entry points is exported (kernels and helpers stay hidden)
    assert exported == set(names)


def test_library_loads_and_reports(lib_path):
    lib = _lib.load(lib_path)
    assert b"sm_100a" in lib.mxb_version()
    for name in _lib.exported_names_from_header():
        assert hasattr(lib, name)


def test_reference_signatures_kept():
    """The drop-ins keep the reference's argument lists (counted from the header)."""
    import re
    text = open(_lib.HEADER).read()

    def nargs(fn):
        m = re.search(r"MXB_API\s+int32_t\s+" + fn + r"\((.*?)\);", text, re.S)
        return len([a for a in m.group(1).split(",") if a.strip()])
    assert nargs("CBHGEMM") == 35        # codeGen/H2GEMM.h:380-389
    assert nargs("blockGEMM") == 33      # codeGen/H2GEMM.h:255-262
    assert nargs("HGEMM") == 32          # symGen/HGEMM_gen.h:120-124
    assert nargs("parHSSGEMM") == 27     # codeGen/HSSGEMM.h:131-134
    assert nargs("seqHSSGEMM") == 25     # codeGen/HSSGEMM.h:18-21
    assert nargs("HGEMM_HSS") == 24      # codeGen/HGEMM_gen.h:120-124


def test_built_for_sm100a(lib_path):
    """The fatbin holds sm_100a code (checked through cuobjdump's element list only)."""
    cuobjdump = "/usr/local/cuda/bin/cuobjdump"
    if not os.path.exists(cuobjdump):
        pytest.skip("cuobjdump not available")
    out = subprocess.run([cuobjdump, "--list-elf", lib_path], capture_output=True, text=True).stdout
    assert "sm_100a" in out


def test_binding_constants_match_header():
    """The Python binding's constants are the header's #defines (error codes, precision modes and
    flags, test hooks, tile and phase codes)."""
    import re
    text = open(_lib.HEADER).read()
    defines = {m.group(1): int(m.group(2), 0)
               for m in re.finditer(r"#define\s+(MXB_[A-Z0-9_]+)\s+\(?(-?(?:0x)?[0-9A-Fa-f]+)\)?", text)}
    pairs = {
        "MXB_OK": _lib.MXB_OK, "MXB_ERR_ARG": _lib.MXB_ERR_ARG, "MXB_ERR_STRUCTURE": _lib.MXB_ERR_STRUCTURE,
        "MXB_ERR_CUDA": _lib.MXB_ERR_CUDA, "MXB_ERR_NOMEM": _lib.MXB_ERR_NOMEM, "MXB_ERR_TIMEOUT": _lib.MXB_ERR_TIMEOUT,
        "MXB_ERR_UNSUPPORTED": _lib.MXB_ERR_UNSUPPORTED, "MXB_CACHE_SAMPLED": _lib.MXB_CACHE_SAMPLED,
        "MXB_CACHE_FULL": _lib.MXB_CACHE_FULL, "MXB_CACHE_OFF": _lib.MXB_CACHE_OFF, "MXB_PREC_FP64": _lib.PREC_FP64,
        "MXB_PREC_SPLIT_BF16": _lib.PREC_SPLIT_BF16, "MXB_PREC_SPLIT_BF16_FAR6": _lib.PREC_SPLIT_BF16_FAR6,
        "MXB_PREC_SPLIT_BF16_X6": _lib.PREC_SPLIT_BF16_X6, "MXB_PLAN_ADJOINT": _lib.PLAN_ADJOINT,
        "MXB_TILE_PAIR": _lib.TILE_PAIR, "MXB_DEBUG_STALL_ONE_WAIT": _lib.DEBUG_STALL_ONE_WAIT,
        "MXB_DEBUG_CHAIN_LEVELS": _lib.DEBUG_CHAIN_LEVELS, "MXB_DEBUG_STALL_LEVEL": _lib.DEBUG_STALL_LEVEL,
        "MXB_DEBUG_ONE_LAUNCH": _lib.DEBUG_ONE_LAUNCH,
    }
    missing = [k for k in pairs if k not in defines]
    assert not missing, missing
    assert {k: defines[k] for k in pairs} == pairs
