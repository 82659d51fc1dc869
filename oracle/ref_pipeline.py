"""ORACLE -- test infrastructure only.

Runs the reference's own host pipeline, built from its sources by ``oracle/Makefile`` into
``oracle/_ref`` (``ref_structure`` and ``ref_cds``), on a points array and loads the CDS it
produces:

1. ``ref_structure``: the reference's structure generator (``sympiler/MatRox.cpp:15-43``):
   cluster tree, budget near / far lists, 32-NN sampling lists, coarsened level sets and
   blocking, written as the reference's ``.bin`` structure files
   (``sympiler/HTree.cpp:469-543``), plus the generated evaluator ``<prefix>_gen.h``;
2. ``ref_cds``: the reference's executor up to the evaluation (``matroxTest-V1/main.cpp:22-92``):
   ``readHtree`` of those files, ID compression with k-NN row sampling
   (``matroxTest-V1/compression.h:1057-1076``) and CDS packing (``DUV2CDS``,
   ``matroxTest-V1/hcds.h:433-460``).  It writes every array the evaluator takes.

The loaded :class:`matrox_ru_b200.structure.CDS` holds the reference's arrays unchanged
(``Dptr`` / ``Bptr`` / ``VTptr`` layouts, ``cidx``, ``wpart`` / ``clevelset`` as
``BalanceCoarLevelSet`` leaves them), so the drop-ins can be checked on what the reference's
``DUV2CDS`` really writes.  Only tests/, the fixture script under tests/golden and bench.py's
checker use this module.
"""
from __future__ import annotations

import dataclasses
import os
import subprocess
import sys
import tempfile
from typing import Dict, Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

STRUCTURE_BIN = os.path.join(HERE, "_ref", "ref_structure")
CDS_BIN = os.path.join(HERE, "_ref", "ref_cds")
_DT = {"f64": np.float64, "u64": np.uint64, "i32": np.int32}


def available() -> bool:
    return os.path.exists(STRUCTURE_BIN) and os.path.exists(CDS_BIN)


@dataclasses.dataclass
class RefRun:
    """One run of the reference pipeline: the CDS, the raw arrays and where the files are."""
    cds: object                      # matrox_ru_b200.structure.CDS
    arrays: Dict[str, np.ndarray]    # every array ref_cds wrote, as written
    scalars: Dict[str, int]
    structure_dir: str               # the reference's .bin structure files
    generated: str                   # path of the generated evaluator (<prefix>_gen.h)
    workdir: str


def _run(cmd, cwd, threads):
    env = dict(os.environ, OMP_NUM_THREADS=str(threads), OPENBLAS_NUM_THREADS="1")
    out = subprocess.run(cmd, cwd=cwd, capture_output=True, text=True, env=env)
    if out.returncode != 0:
        raise RuntimeError(f"{os.path.basename(cmd[0])} failed ({out.returncode}):\n{out.stdout}\n{out.stderr}")
    return out.stdout


def read_dump(outdir: str):
    arrays, scalars = {}, {}
    with open(os.path.join(outdir, "meta.txt")) as f:
        for line in f:
            kind, name, *rest = line.split()
            if kind == "scalar":
                scalars[name] = int(rest[0])
            else:
                dt, count = _DT[rest[0]], int(rest[1])
                a = np.fromfile(os.path.join(outdir, name + ".bin"), dtype=dt)
                if a.size != count:
                    raise ValueError(f"{name}: {a.size} values, meta says {count}")
                arrays[name] = a
    return arrays, scalars


def cds_from_dump(arrays, scalars):
    """The reference's hcds / HTree arrays as a structure.CDS (no array is re-packed)."""
    from matrox_ru_b200 import structure as S
    nn, nl = scalars["numnodes"], scalars["nleaf"]
    hss = bool(scalars["is_hss"])
    lids, lofs_node, lens = arrays["lids"], arrays["lidsoffset"], arrays["lidslen"]
    leaf = arrays["leaf"]
    perm = np.concatenate([lids[lofs_node[leaf[i]]:lofs_node[leaf[i]] + lens[leaf[i]]]
                           for i in range(nl)]).astype(np.int64)
    Ddim = arrays["Ddim"]
    lofs = np.concatenate([[0], np.cumsum(Ddim.astype(np.int64))]).astype(np.int64)
    slen = arrays["slen"]
    skels, off = [np.zeros(0, np.int64)], 0
    for v in range(1, nn):
        skels.append(arrays["skels"][off:off + slen[v]].astype(np.int64))
        off += int(slen[v])
    z = np.zeros(1, np.int32)
    return S.CDS(n=scalars["n"], nleaf=nl, numnodes=nn, depth=scalars["depth"], is_hss=hss,
                 D=arrays["D"], Dptr=arrays["Dptr"], B=arrays["B"], Bptr=arrays["Bptr"],
                 VT=arrays["VT"], VTptr=arrays["VTptr"], lchildren=arrays["lchildren"],
                 rchildren=arrays["rchildren"], levelset=arrays["levelset"], idx=arrays["idx"],
                 Ddim=Ddim, lm=arrays["lm"], slen=slen,
                 nblockset=arrays.get("nblockset", z), nblocks=arrays.get("nblocks", z),
                 npairx=arrays["npairx"], npairy=arrays["npairy"],
                 fblockset=arrays.get("fblockset", z), fblocks=arrays.get("fblocks", z),
                 fpairx=arrays["fpairx"], fpairy=arrays["fpairy"], wpart=arrays["wpart"],
                 clevelset=arrays["clevelset"], cidx=arrays["cidx"], perm=perm,
                 leaf_lids_offset=lofs, skels=skels)


def run(X: np.ndarray, *, budget: float, leaf: int, tol: float, h: float, max_rank: int,
        samples: Optional[int] = None, threads: int = 1, workdir: Optional[str] = None) -> RefRun:
    """Reference structure + compression + CDS for points X (n x d), Gaussian kernel with
    bandwidth h.  ``samples`` is the reference's ``m`` of ``compression`` (default: leaf).
    One thread reproduces the reference's rand()-based sampling exactly from run to run."""
    if not available():
        raise FileNotFoundError("oracle/_ref/ref_structure and ref_cds are not built "
                                "(oracle/Makefile with REF_ROOT set to the reference tree)")
    X = np.ascontiguousarray(X, dtype=np.float64)
    n, d = X.shape
    work = workdir or tempfile.mkdtemp(prefix="mxb_refpipe_")
    sdir, edir, odir = (os.path.join(work, s) for s in ("sympiler", "exec", "cds"))
    for p in (sdir, edir, odir):
        os.makedirs(p, exist_ok=True)
    pts = os.path.join(work, "points.bin")
    X.tofile(pts)
    _run([STRUCTURE_BIN, pts, str(n), str(d), repr(float(budget)), str(leaf), os.path.join(sdir, "HGEMM")],
         sdir, threads)
    hss = not os.path.exists(os.path.join(sdir, "nblockset.bin"))
    _run([CDS_BIN, pts, str(n), str(d), repr(float(tol)), repr(float(h)), str(max_rank),
          str(samples or leaf), "1" if hss else "0", odir], edir, threads)
    arrays, scalars = read_dump(odir)
    return RefRun(cds=cds_from_dump(arrays, scalars), arrays=arrays, scalars=scalars,
                  structure_dir=sdir, generated=os.path.join(sdir, "HGEMM_gen.h"), workdir=work)
