"""Generates the reference-pipeline fixtures ``tests/golden/ref_pipeline/*.npz``.

Unlike ``make_golden.py``, whose CDSs come from this repository's producer, these fixtures
hold a CDS made end to end by the REFERENCE's own host code, built from its sources by
``oracle/Makefile`` (``oracle/_ref/ref_structure`` and ``ref_cds``, driven by
``oracle/ref_pipeline.py``):

* the structure generator's ``.bin`` files (``sympiler/HTree.cpp:469-543``) and k-NN lists;
* every array of the reference's CDS as ``DUV2CDS`` / ``BalanceCoarLevelSet`` leave them
  (``matroxTest-V1/hcds.h:433-460``, ``compression.h:1003-1076``);
* a right-hand side TW (leaf-blocked) and the outputs of three reference evaluators on it:
  - ``Y_generated``: the evaluator the generator emitted for this very structure
    (``<prefix>_gen.h``, the code matroxTest-V1/main.cpp:97-107 calls), compiled here;
  - ``Y_structure_generic``: the reference's ``CBHGEMM`` / ``parHSSGEMM``
    (``codeGen/H2GEMM.h:380``, ``codeGen/HSSGEMM.h:131``, from ``oracle/_ref/libmatrox_ref.so``).

Run from the repository root where the reference tree is present:

    make -C oracle REF_ROOT=<reference tree> && python tests/golden/make_ref_pipeline.py <reference tree>

The reference samples with rand() inside OpenMP loops, so the pipeline runs on one thread.
"""
import ctypes
import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle")]

from matrox_ru_b200 import structure as S  # noqa: E402
import oracle as O  # noqa: E402
import ref_pipeline as RP  # noqa: E402

CASES = {
    # name: (n, d, components, mean_lo, mean_hi, sigma, seed, budget, leaf, tol, h, max_rank, nrhs)
    "hss_n1024": (1024, 8, 8, 0.0, 4.0, 0.5, 201, 0.0, 32, 1e-5, 1.0, 24, 5),
    "h2b_n1024": (1024, 8, 8, 0.0, 4.0, 0.5, 202, 0.12, 32, 1e-5, 1.0, 24, 4),
}

# One C++ translation unit around the generated evaluator: the generated header defines
# HGEMM with C linkage and includes the reference's <cholUtils.h> (symGen/).
_WRAP = '#include "{gen}"\n'


def compile_generated(gen_header: str, ref_root: str, workdir: str) -> ctypes.CDLL:
    src = os.path.join(workdir, "gen_wrap.cpp")
    with open(src, "w") as f:
        f.write(_WRAP.format(gen=gen_header))
    so = os.path.join(workdir, "libgen.so")
    shim = os.path.join(ROOT, "oracle", "mkl_shim")
    oblas = [p for p in (os.path.join(os.path.dirname(np.__file__), "..", "scipy.libs"),) if os.path.isdir(p)]
    libdir = os.path.realpath(oblas[0])
    lib = [f for f in os.listdir(libdir) if f.startswith("libscipy_openblas")][0]
    cmd = ["g++", "-O0", "-fopenmp", "-fPIC", "-shared", "-w", "-include", "cstdint", "-I", shim,
           "-I", os.path.join(ref_root, "symGen"), "-o", so, src, "-L", libdir, "-l:" + lib,
           "-Wl,-rpath," + libdir]
    out = subprocess.run(cmd, capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("compiling the generated evaluator failed:\n" + out.stderr)
    return ctypes.CDLL(so)


def run_generated(lib, run, TW, r):
    """Calls the generated HGEMM as matroxTest-V1/main.cpp:97-107 does (idx = cidx, the
    reference's own offsets for r right-hand sides, zeroed workspaces and apres)."""
    a, cds = run.arrays, run.cds
    keep = []

    def p(x, dt=np.int32):
        x = np.ascontiguousarray(x if np.asarray(x).size else np.zeros(1, dt), dtype=dt)
        keep.append(x)
        return x.ctypes.data_as(ctypes.c_void_p)

    wptr = a["wptr1"].astype(np.int64) * r
    wsko = a["wskeloffset1"].astype(np.int64) * r
    nskel = int(cds.slen.astype(np.int64).sum()) * r
    wskel, uskel = np.zeros(max(nskel, 1)), np.zeros(max(nskel, 1))
    TW = np.ascontiguousarray(TW, dtype=np.float64)
    Y = np.zeros_like(TW)
    args = [p(cds.D, np.float64), p(cds.B, np.float64), p(cds.VT, np.float64), p(cds.Dptr, np.uint64),
            p(cds.Bptr, np.uint64), p(cds.VTptr), p(cds.lchildren), p(cds.rchildren), p(cds.levelset),
            p(cds.cidx), TW.ctypes.data_as(ctypes.c_void_p), Y.ctypes.data_as(ctypes.c_void_p),
            ctypes.c_int32(r), p(cds.Ddim), p(wptr), p(wptr), wskel.ctypes.data_as(ctypes.c_void_p),
            p(wsko), uskel.ctypes.data_as(ctypes.c_void_p), p(wsko), p(cds.lm), p(cds.slen)]
    if not cds.is_hss:
        args += [p(cds.nblockset), p(cds.nblocks), p(cds.npairx), p(cds.npairy), p(cds.fblockset),
                 p(cds.fblocks), p(cds.fpairx), p(cds.fpairy)]
    args += [p(cds.wpart), p(cds.clevelset)]
    lib.HGEMM.restype = ctypes.c_int32
    lib.HGEMM(*args)
    return Y


def main():
    if len(sys.argv) != 2:
        raise SystemExit(__doc__)
    ref_root = sys.argv[1]
    if not (RP.available() and O.ref_available()):
        raise SystemExit("oracle/_ref is not built: make -C oracle REF_ROOT=<reference tree>")
    out_dir = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ref_pipeline")
    os.makedirs(out_dir, exist_ok=True)
    for name, (n, d, k, lo, hi, sig, seed, budget, leaf, tol, h, mr, r) in CASES.items():
        X = S.gaussian_mixture(n, d, k, lo, hi, sig, None, seed)
        work = tempfile.mkdtemp(prefix="mxb_fixture_")
        run = RP.run(X, budget=budget, leaf=leaf, tol=tol, h=h, max_rank=mr, threads=1, workdir=work)
        cds = run.cds
        TW = np.random.default_rng(seed).standard_normal(n * r)
        Yg = run_generated(compile_generated(run.generated, ref_root, work), run, TW, r)
        Ys = O.eval_h2b(cds, TW, r, use_reference=True)
        gap = np.abs(Yg - Ys).max() / np.abs(Ys).max()
        if not gap <= 1e-12:
            raise SystemExit(f"{name}: the generated and the structure-generic reference evaluators differ ({gap:.2e})")
        z = {"X": X, "TW": TW, "Y_generated": Yg, "Y_structure_generic": Ys, "nrhs": np.array([r]),
             "params": np.array([budget, leaf, tol, h, mr], np.float64)}
        for f in sorted(os.listdir(run.structure_dir)):
            if f.endswith(".bin"):
                dt = "<f8" if f == "distNN.bin" else "<i4"
                z["struct/" + f] = np.fromfile(os.path.join(run.structure_dir, f), dtype=dt)
        for key, v in run.arrays.items():
            z["cds/" + key] = v
        z["scalars"] = np.array([[key, v] for key, v in run.scalars.items()], dtype=object).astype(str)
        path = os.path.join(out_dir, name + ".npz")
        np.savez_compressed(path, **z)
        print(name, "hss" if cds.is_hss else "h2b", "nleaf", cds.nleaf, "near", cds.ncount, "far", cds.fcount,
              "generated vs CBHGEMM/parHSSGEMM %.1e" % gap, "bytes", os.path.getsize(path))


if __name__ == "__main__":
    main()
