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
