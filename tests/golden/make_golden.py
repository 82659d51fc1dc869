"""Generates the golden fixtures of tests/golden from the REFERENCE's own evaluator.

Each fixture holds a small CDS (built by matrox_ru_b200.structure), a right-hand side TW in
the leaf-blocked layout and the output of the reference's compiled CBHGEMM / parHSSGEMM
(codeGen/H2GEMM.h:380, codeGen/HSSGEMM.h:131, built by oracle/Makefile into oracle/_ref)
on those arrays.  Run from the repository root where the reference tree is available:

    make -C oracle && python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle")]

from matrox_ru_b200 import structure as S  # noqa: E402
import oracle as O  # noqa: E402

CASES = {
    # name: (n, d, comps, lo, hi, sig_lo, sig_hi, seed, kernel, h, leaf, budget, tol, max_rank, nrhs)
    "hss_n256": (256, 3, 3, 0.0, 2.0, 0.4, None, 101, "gaussian", 1.0, 16, 0.0, 1e-6, 12, 5),
    "h2b_n384": (384, 4, 4, 0.0, 3.0, 0.4, None, 102, "gaussian", 1.0, 24, 0.25, 1e-6, 16, 3),
    "h2b_ragged_n300": (300, 3, 3, -1.0, 1.0, 0.3, 0.7, 103, "imq", 1.0, 20, 0.3, 1e-5, 12, 4),
}


def main():
    if not O.ref_available():
        raise SystemExit("oracle/_ref/libmatrox_ref.so missing: run `make -C oracle` with the reference tree present")
    out_dir = os.path.dirname(os.path.abspath(__file__))
    for name, (n, d, k, lo, hi, sl, sh, seed, kind, h, leaf, budget, tol, mr, r) in CASES.items():
        X = S.gaussian_mixture(n, d, k, lo, hi, sl, sh, seed)
        cds = S.build_cds(X, S.KernelSpec(kind, h), leaf_size=leaf, budget=budget, tol=tol, max_rank=mr, seed=seed)
        rng = np.random.default_rng(seed)
        TW = rng.standard_normal(n * r)
        Y0 = np.zeros(n * r) if cds.is_hss else rng.standard_normal(n * r)  # H2-b accumulates
        Y = O.eval_h2b(cds, TW, r, Y=Y0.copy(), use_reference=True)
        path = os.path.join(out_dir, f"{name}.npz")
        cds.save(path)
        z = dict(np.load(path))
        z.update(X=X, TW=TW, Y0=Y0, Yref=Y, nrhs=np.array([r]))
        np.savez_compressed(path, **z)
        print(name, "hss" if cds.is_hss else "h2b", "nleaf", cds.nleaf, "near", cds.ncount, "far", cds.fcount,
              "bytes", os.path.getsize(path))


if __name__ == "__main__":
    main()
