"""ORACLE -- test infrastructure only.

Compression quality of the reference's own host pipeline against this repository's CDS
producer (``matrox_ru_b200.structure.build_cds``) on the same points: for each, the relative
error of the FP64 evaluation (the oracle's restatement, checked against the reference
evaluator on both CDSs) against the dense FP64 K W on sampled rows, with the ranks and list
sizes.  The two differ in how the ID samples rows: the reference takes the 32-NN lists
(``matroxTest-V1/compression.h:362-443``) plus uniform random rows; the producer here takes
nearest outside points of neighbouring leaves plus uniform random rows.

    python oracle/compare_compression.py c0|c1 [--threads T] [--nrhs R]

c0: HSS, N=16384, d=8, 8-component mixture (means U[0,4]^8, sigma 0.5), h=1.0, leaf 128,
    tolerance 1e-5, max rank 128.
c1: H2-b, N=65536, d=28, 16 components (means U[-2,2]^28, sigma U[0.3,1.0]), h=2.0, leaf 256,
    budget 0.03, tolerance 1e-5, max rank 256.
"""
import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [os.path.dirname(HERE), HERE]

from matrox_ru_b200 import structure as S  # noqa: E402
import oracle as O  # noqa: E402
import ref_pipeline as RP  # noqa: E402

CONFIGS = {
    "c0": dict(n=16384, d=8, comps=8, lo=0.0, hi=4.0, slo=0.5, shi=None, seed=20261202, h=1.0, leaf=128,
               budget=0.0, tol=1e-5, max_rank=128),
    "c1": dict(n=65536, d=28, comps=16, lo=-2.0, hi=2.0, slo=0.3, shi=1.0, seed=20261203, h=2.0, leaf=256,
               budget=0.03, tol=1e-5, max_rank=256),
}


def dense_error(cds, X, spec, r, rows, W):
    TW = cds.to_tree_order(W).reshape(-1)
    Y = cds.from_tree_order(O.eval_h2b(cds, TW, r), r)
    dense = S.dense_kernel_times(X, W, spec, rows=rows)
    ref_gap = None
    if O.ref_available():
        Yr = O.eval_h2b(cds, TW, r, use_reference=True)
        ref_gap = float(np.abs(Yr - cds.to_tree_order(Y).reshape(-1)).max() / np.abs(Yr).max())
    return float(np.linalg.norm(Y[rows] - dense) / np.linalg.norm(dense)), ref_gap


def describe(cds):
    s = cds.slen[1:]
    return dict(ranks_min_median_max=[int(s.min()), int(np.median(s)), int(s.max())], near_pairs=int(cds.ncount),
                far_pairs=int(cds.fcount), nleaf=int(cds.nleaf))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("config", choices=sorted(CONFIGS))
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--nrhs", type=int, default=16)
    a = ap.parse_args()
    c = CONFIGS[a.config]
    X = S.gaussian_mixture(c["n"], c["d"], c["comps"], c["lo"], c["hi"], c["slo"], c["shi"], seed=c["seed"])
    spec = S.KernelSpec("gaussian", c["h"])
    r = a.nrhs
    W = np.random.default_rng(c["seed"] + 1).standard_normal((c["n"], r))
    rows = np.random.default_rng(0).choice(c["n"], 64, replace=False)
    out = {"config": a.config, "nrhs": r, "rows": 64}
    t = time.time()
    run = RP.run(X, budget=c["budget"], leaf=c["leaf"], tol=c["tol"], h=c["h"], max_rank=c["max_rank"],
                 threads=a.threads)
    out["reference_pipeline_s"] = round(time.time() - t, 1)
    e, gap = dense_error(run.cds, X, spec, r, rows, W)
    out["reference_cds"] = dict(describe(run.cds), rel_err_vs_dense=e, oracle_vs_reference_evaluator=gap)
    t = time.time()
    ours = S.build_cds(X, spec, leaf_size=c["leaf"], budget=c["budget"], tol=c["tol"], max_rank=c["max_rank"],
                       seed=c["seed"])
    out["repository_producer_s"] = round(time.time() - t, 1)
    e, gap = dense_error(ours, X, spec, r, rows, W)
    out["repository_cds"] = dict(describe(ours), rel_err_vs_dense=e, oracle_vs_reference_evaluator=gap)
    print(json.dumps(out))


if __name__ == "__main__":
    main()
