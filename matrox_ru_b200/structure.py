"""Host-side producer of the compressed data storage (CDS) that the evaluator consumes.

MatRox splits its pipeline in two: host code builds the cluster tree, the near/far
interaction lists, the blocked and coarsened schedules and the interpolative
decomposition (ID) in FP64, and packs the result into flat arrays (the CDS); the
evaluator ``HGEMM`` then computes ``Y = K~ W`` from those arrays.  This module is the
host half, restated so that the evaluator can be fed without the reference's
Sympiler code generator.  It produces arrays in exactly the layout the reference's
``HGEMM`` reads (names follow ``matroxTest-V1/hcds.h:10-34`` and
``matroxTest-V1/HTree.h:17-74``):

* tree: heap-numbered perfect binary tree, root 0, children ``2v+1``/``2v+2``; points
  split by projection on the farthest-pair direction at the median
  (``sympiler/boundingbox.cpp:337-449``, ``sympiler/ClusterTree.cpp:81-241``);
* near lists with a budget (``ClusterTree.cpp:508-576``), far lists by recursive
  admissibility against the near lists then merged bottom-up
  (``ClusterTree.cpp:629-684``);
* blocked near (rows of 2 leaves) and far (rows of 4 nodes) CSR-of-CSR lists
  (``ClusterTree.cpp:951-1089``, ``sympiler/HTree.cpp:83-166``);
* coarsened level sets ``parlevel(2,2)`` with post-order partitions
  (``ClusterTree.cpp:732-857``, ``sympiler/DSInspector.cpp:64-160``);
* ID by column-pivoted QR with the reference's rank rule
  (``matroxTest-V1/compression.h:446-523``) on sampled kernel rows
  (``compression.h:597-797``);
* packing of near blocks ``D``, far couplings ``B`` and projections ``VT``
  (``matroxTest-V1/hcds.h:339-763``).

ID rows are sampled as the reference samples them: k-NN sampling and pruning neighbours
(``compression.h:362-443``) on 32-NN lists (the reference generator's own lists when a
structure read from its files carries them, else exact lists laid out as the reference's
max-heaps), then uniform random points.  The tree split fills a perfect tree (every level
split) so the heap numbering the reference assumes always holds.
"""
from __future__ import annotations

import contextlib
import dataclasses
import math
import os
from concurrent.futures import ThreadPoolExecutor
from typing import Dict, List, Optional, Tuple

import numpy as np

try:  # scipy provides LAPACK dgeqp3 through qr(pivoting=True)
    import scipy.linalg as _sla
except Exception as exc:  # pragma: no cover - scipy is part of the image
    raise ImportError("matrox_ru_b200.structure needs scipy for the ID compression") from exc


# ---------------------------------------------------------------------------
# kernels
# ---------------------------------------------------------------------------

@dataclasses.dataclass(frozen=True)
class KernelSpec:
    """Kernel function k(x, y) of the compressed matrix.

    ``gaussian``: exp(-|x-y|^2 / (2 h^2))  (``matroxTest-V1/compression.h:41-100``)
    ``imq``:      1 / sqrt(1 + |x-y|^2 / h^2)  (inverse multiquadric)
    ``newton``:   1 / |x-y|, with 1 on the diagonal (``compression.h:112-131``)
    """

    kind: str = "gaussian"
    h: float = 1.0

    def __post_init__(self):
        if self.kind not in ("gaussian", "imq", "newton"):
            raise ValueError(f"unknown kernel kind {self.kind!r}")
        if not (self.h > 0):
            raise ValueError("kernel bandwidth h must be positive")


def sqdist(A: np.ndarray, B: np.ndarray) -> np.ndarray:
    """Squared distances |a_i - b_j|^2 via |a|^2 + |b|^2 - 2 a.b, clamped at 0."""
    d2 = (A * A).sum(1)[:, None] + (B * B).sum(1)[None, :] - 2.0 * (A @ B.T)
    np.maximum(d2, 0.0, out=d2)
    return d2


def kernel_matrix(X: np.ndarray, rows, cols, spec: KernelSpec) -> np.ndarray:
    """Dense kernel block K(X[rows], X[cols]) in FP64 (C-ordered, rows x cols).

    The Gaussian and the inverse multiquadric take squared distances from the norm expansion
    (as the reference's Gaussian does, ``compression.h:256-300``).  The 1/r kernel sums the
    squared coordinate differences, as the reference does (``compression.h:338-350``), so
    coincident points give exactly 0 and the value 1."""
    if spec.kind == "newton":
        A, B = X[rows], X[cols]
        d2 = np.zeros((len(A), len(B)))
        for k in range(X.shape[1]):
            diff = A[:, k][:, None] - B[:, k][None, :]
            d2 += diff * diff
        r = np.sqrt(d2)
        r[r == 0] = 1.0
        return 1.0 / r
    d2 = sqdist(X[rows], X[cols])
    if spec.kind == "gaussian":
        return np.exp(d2 * (-0.5 / (spec.h * spec.h)))
    return 1.0 / np.sqrt(1.0 + d2 / (spec.h * spec.h))


# ---------------------------------------------------------------------------
# synthetic point sets
# ---------------------------------------------------------------------------

def gaussian_mixture(n: int, d: int, components: int, mean_lo: float, mean_hi: float,
                     sigma_lo: float, sigma_hi: Optional[float], seed: int) -> np.ndarray:
    """Seeded isotropic Gaussian mixture, N x d row-major FP64.

    Component means are uniform in [mean_lo, mean_hi]^d, each component's sigma is
    ``sigma_lo`` (or uniform in [sigma_lo, sigma_hi]); points are assigned to
    components uniformly.
    """
    rng = np.random.default_rng(seed)
    means = rng.uniform(mean_lo, mean_hi, size=(components, d))
    if sigma_hi is None:
        sig = np.full(components, float(sigma_lo))
    else:
        sig = rng.uniform(sigma_lo, sigma_hi, size=components)
    lab = rng.integers(0, components, size=n)
    X = means[lab] + rng.standard_normal((n, d)) * sig[lab][:, None]
    return np.ascontiguousarray(X, dtype=np.float64)


# ---------------------------------------------------------------------------
# tree
# ---------------------------------------------------------------------------

def _split(X: np.ndarray, ids: np.ndarray) -> Tuple[np.ndarray, np.ndarray]:
    """Split ``ids`` in two halves by projection on the farthest-pair direction.

    Follows ``sympiler/boundingbox.cpp:337-449``: x0 = farthest point from the mean,
    x1 = farthest point from x0, project on x1 - x0, left gets the ceil(n/2) smallest.
    """
    P = X[ids]
    c = P.mean(0)
    x0 = int(np.argmax(((P - c) ** 2).sum(1)))
    x1 = int(np.argmax(((P - P[x0]) ** 2).sum(1)))
    proj = P @ (P[x1] - P[x0])
    order = np.argsort(proj, kind="stable")
    nl = (len(ids) + 1) // 2
    return ids[order[:nl]], ids[order[nl:]]


@dataclasses.dataclass
class Tree:
    depth: int                 # number of split levels; leaves sit at this level
    numnodes: int
    nleaf: int
    lids: List[np.ndarray]     # point ids per node
    mid: np.ndarray            # nleaf x d bounding-box mid points of the leaves
    radius: np.ndarray         # nleaf half-diagonals of the leaf boxes

    @property
    def first_leaf(self) -> int:
        return (1 << self.depth) - 1

    def is_leaf(self, v: int) -> bool:
        return v >= self.first_leaf

    def level(self, v: int) -> int:
        return int(math.floor(math.log2(v + 1)))

    def parent(self, v: int) -> int:
        return (v - 1) // 2

    def leaf_index(self, v: int) -> int:
        return v - self.first_leaf

    def leaf_node(self, i: int) -> int:
        return i + self.first_leaf

    def leaf_range(self, v: int) -> Tuple[int, int]:
        """Leaf indices [lo, hi) below node v."""
        lv = self.level(v)
        span = 1 << (self.depth - lv)
        first_at_level = (1 << lv) - 1
        lo = (v - first_at_level) * span
        return lo, lo + span


def build_tree(X: np.ndarray, leaf_size: int) -> Tree:
    n = X.shape[0]
    if n < 1:
        raise ValueError("need at least one point")
    depth = 0
    while (n >> depth) > leaf_size and (n >> (depth + 1)) >= 1:
        depth += 1
    # ceil division check: every leaf must hold <= leaf_size points
    while math.ceil(n / (1 << depth)) > leaf_size:
        depth += 1
    if (1 << depth) > n:
        raise ValueError("leaf_size too small for the number of points")
    numnodes = (1 << (depth + 1)) - 1
    lids: List[Optional[np.ndarray]] = [None] * numnodes
    lids[0] = np.arange(n, dtype=np.int64)
    for v in range((1 << depth) - 1):
        a, b = _split(X, lids[v])
        lids[2 * v + 1] = a
        lids[2 * v + 2] = b
    first = (1 << depth) - 1
    nleaf = 1 << depth
    mids = np.empty((nleaf, X.shape[1]))
    rads = np.empty(nleaf)
    for i in range(nleaf):
        P = X[lids[first + i]]
        lo, hi = P.min(0), P.max(0)
        mids[i] = 0.5 * (lo + hi)
        rads[i] = np.sqrt(((hi - mids[i]) ** 2).sum())
    return Tree(depth, numnodes, nleaf, lids, mids, rads)


# ---------------------------------------------------------------------------
# interaction lists
# ---------------------------------------------------------------------------

def near_lists(tree: Tree, budget: float) -> List[List[int]]:
    """Near leaves (leaf indices) of every leaf, sorted ascending, self included.

    Budget rule of ``sympiler/ClusterTree.cpp:508-576``: leaves are ranked by
    |mid_i - mid_j| / (r_i + r_j); after self, the next ones are added while the list
    is shorter than int(nleaf * budget - 1).  budget 0 gives HSS (self only).
    """
    nl = tree.nleaf
    cap = int(nl * budget - 1)
    out = []
    if nl == 1:
        return [[0]]
    d = np.sqrt(sqdist(tree.mid, tree.mid))
    rs = tree.radius[:, None] + tree.radius[None, :]
    with np.errstate(divide="ignore", invalid="ignore"):
        ratio = np.where(rs > 0, d / rs, np.where(d > 0, np.inf, 0.0))
    for i in range(nl):
        order = [j for j in np.argsort(ratio[i], kind="stable") if j != i]
        lst = [i]
        for j in order:
            if len(lst) < cap:
                lst.append(int(j))
            else:
                break
        out.append(sorted(lst))
    return out


def far_lists(tree: Tree, near: List[List[int]]) -> List[List[int]]:
    """Far nodes of every node (node ids), sorted ascending.

    For every leaf, the tree is walked from the root: a subtree holding none of the
    leaf's near leaves is far, otherwise its children are visited
    (``ClusterTree.cpp:665-704``).  Then, bottom-up, far nodes shared by both
    children move to the parent (``ClusterTree.cpp:629-662``).
    """
    far: List[List[int]] = [[] for _ in range(tree.numnodes)]
    if tree.depth == 0:
        return far

    def contains_near(root: int, nset: List[int]) -> bool:
        lo, hi = tree.leaf_range(root)
        return any(lo <= j < hi for j in nset)

    for i in range(tree.nleaf):
        v = tree.leaf_node(i)
        nset = near[i]
        stack = [0]
        found = []
        # preorder, left before right
        def walk(root):
            if contains_near(root, nset):
                if not tree.is_leaf(root):
                    walk(2 * root + 1)
                    walk(2 * root + 2)
            else:
                found.append(root)
        walk(0)
        far[v] = found
    for lev in range(tree.depth - 1, 0, -1):
        for v in range((1 << lev) - 1, (1 << (lev + 1)) - 1):
            lc, rc = 2 * v + 1, 2 * v + 2
            rset = set(far[rc])
            common = [w for w in far[lc] if w in rset]
            if common:
                cset = set(common)
                far[v].extend(common)
                far[lc] = [w for w in far[lc] if w not in cset]
                far[rc] = [w for w in far[rc] if w not in cset]
    return [sorted(f) for f in far]


def node_order_bottom_up(tree: Tree) -> List[int]:
    """Non-root nodes level by level from the leaves up, ascending inside a level
    (``ClusterTree.cpp:1095-1107``, ``nodeId``)."""
    out = []
    for lev in range(tree.depth, 0, -1):
        out.extend(range((1 << lev) - 1, (1 << (lev + 1)) - 1))
    return out


def blocked_near(tree: Tree, near: List[List[int]], block: int = 2):
    """CSR-of-CSR near blocking (``ClusterTree.cpp:951-1017``, ``HTree.cpp:83-124``)."""
    nl = tree.nleaf
    nrow = (nl - 1 + block) // block
    rows: List[Dict[int, List[Tuple[int, int]]]] = [dict() for _ in range(nrow)]
    for x in range(nl):
        r = x // block
        for y in near[x]:
            rows[r].setdefault(y // block, []).append((x, y))
    nblockset = [0]
    nblocks = [0]
    px, py = [], []
    for r in range(nrow):
        cols = sorted(rows[r].keys())
        for c in cols:
            for (x, y) in rows[r][c]:
                px.append(x)
                py.append(y)
            nblocks.append(len(px))
        nblockset.append(len(nblocks) - 1)
    return (np.array(nblockset, np.int32), np.array(nblocks, np.int32),
            np.array(px, np.int32), np.array(py, np.int32))


def blocked_far(tree: Tree, far: List[List[int]], block: int = 4):
    """CSR-of-CSR far blocking over the bottom-up node order
    (``ClusterTree.cpp:1020-1089``, ``HTree.cpp:126-166``)."""
    order = node_order_bottom_up(tree)
    pos = {v: i for i, v in enumerate(order)}
    nn = len(order)
    nrow = (nn - 1 + block) // block if nn > 0 else 0
    rows: List[Dict[int, List[Tuple[int, int]]]] = [dict() for _ in range(nrow)]
    for v in order:
        r = pos[v] // block
        for w in far[v]:
            rows[r].setdefault(pos[w] // block, []).append((v, w))
    fblockset = [0]
    fblocks = [0]
    px, py = [], []
    for r in range(nrow):
        for c in sorted(rows[r].keys()):
            for (v, w) in rows[r][c]:
                px.append(v)
                py.append(w)
            fblocks.append(len(px))
        fblockset.append(len(fblocks) - 1)
    return (np.array(fblockset, np.int32), np.array(fblocks, np.int32),
            np.array(px, np.int32), np.array(py, np.int32))


def coarsened_levels(tree: Tree, agg: int = 2, llevel: int = 2):
    """Coarsened level sets with post-order partitions, ``parlevel(2,2)`` +
    ``genpostw`` (``ClusterTree.cpp:732-789``, ``DSInspector.cpp:122-160``).

    Returns (clevelset, wpart, cidx): coarse level i owns partitions
    [clevelset[i], clevelset[i+1]); partition k owns cidx[wpart[k]:wpart[k+1]],
    a post-order (children first) of a subtree cut at the coarse level's bottom.
    Level 0 is the bottom (leaves); the root is excluded.
    """
    nlev = tree.depth  # levels below the root, numbered bottom-up 0..depth-1
    if nlev == 0:
        return np.zeros(1, np.int32), np.zeros(1, np.int32), np.zeros(0, np.int32)
    llevel = min(llevel, nlev)
    groups = [list(range(llevel))]
    cur: List[int] = []
    for lv in range(llevel, nlev):
        cur.append(lv)
        if len(cur) == agg:
            groups.append(cur)
            cur = []
    if cur:
        groups.append(cur)

    def tree_level(bl):  # bottom-up level index -> heap level
        return tree.depth - bl

    clevelset = [0]
    wpart = [0]
    cidx: List[int] = []
    for g in groups:
        top, bot = tree_level(g[-1]), tree_level(g[0])
        for v in range((1 << top) - 1, (1 << (top + 1)) - 1):
            part: List[int] = []

            def post(u, lev):
                if lev < bot:
                    post(2 * u + 1, lev + 1)
                    post(2 * u + 2, lev + 1)
                part.append(u)
            post(v, top)
            cidx.extend(part)
            wpart.append(len(cidx))
        clevelset.append(len(wpart) - 1)
    return np.array(clevelset, np.int32), np.array(wpart, np.int32), np.array(cidx, np.int32)


def levelsets_top_down(tree: Tree):
    """levelset / idx without coarsening: levels from the root's children down to the
    leaves, root excluded (``sympiler/HTree.cpp:348-367``)."""
    levelset = [0]
    idx: List[int] = []
    for lev in range(1, tree.depth + 1):
        idx.extend(range((1 << lev) - 1, (1 << (lev + 1)) - 1))
        levelset.append(len(idx))
    return np.array(levelset, np.int32), np.array(idx, np.int32)


# ---------------------------------------------------------------------------
# interpolative decomposition
# ---------------------------------------------------------------------------

def interpolative_decomposition(A: np.ndarray, tol: float, max_rank: int):
    """Column ID of A (rows = samples, cols = candidates), ``compression.h:446-523``.

    Pivoted QR; the rank s is the first s >= 1 with |R[s,s] / R[0,0]| < tol, capped at
    max_rank; the projection P (s x ncols) solves R11 P[:, piv] = R[:s, :].  A zero matrix
    (R[0,0] == 0) gets P = 0, as the reference returns R's (zero) upper rows unsolved there.
    Returns (skeleton column positions, P).
    """
    ncols = A.shape[1]
    R, piv = _sla.qr(A, mode="r", pivoting=True, check_finite=False)
    r00 = R[0, 0] if R.shape[0] > 0 else 0.0
    s = 1
    while s < ncols:
        if s > max_rank:
            break
        rss = R[s, s] if s < R.shape[0] else 0.0
        if r00 != 0 and abs(rss / r00) < tol:
            break
        s += 1
    s = min(s, max_rank, ncols)
    if r00 == 0:
        return piv[:s].copy(), np.zeros((s, ncols))
    T = _sla.solve_triangular(R[:s, :s], R[:s, :], lower=False, check_finite=False)
    P = np.empty((s, ncols))
    P[:, piv] = T
    return piv[:s].copy(), P


# ---------------------------------------------------------------------------
# CDS container
# ---------------------------------------------------------------------------

@dataclasses.dataclass
class CDS:
    """The compressed matrix in the reference's array layout, independent of nrhs.

    Per-nrhs offsets (``wptr/uptr``, ``wskeloffset/uskeloffset``) come from
    :meth:`offsets`.  All index arrays are int32 except ``Dptr``/``Bptr`` (uint64).
    """
    n: int
    nleaf: int
    numnodes: int
    depth: int
    is_hss: bool
    D: np.ndarray          # float64, near blocks, column-major m_x x m_y each
    Dptr: np.ndarray       # uint64 per near pair
    B: np.ndarray          # float64, far couplings, column-major s_x x s_y each
    Bptr: np.ndarray       # uint64 per far pair
    VT: np.ndarray         # float64, projections, column-major s_v x ncols_v each
    VTptr: np.ndarray      # int32 per node
    lchildren: np.ndarray
    rchildren: np.ndarray
    levelset: np.ndarray   # top-down, root excluded
    idx: np.ndarray
    Ddim: np.ndarray       # points per leaf
    lm: np.ndarray         # node -> leaf index or -1
    slen: np.ndarray       # skeleton rank per node (root 0)
    nblockset: np.ndarray
    nblocks: np.ndarray
    npairx: np.ndarray     # near pairs, leaf indices
    npairy: np.ndarray
    fblockset: np.ndarray
    fblocks: np.ndarray
    fpairx: np.ndarray     # far pairs, node ids
    fpairy: np.ndarray
    wpart: np.ndarray
    clevelset: np.ndarray
    cidx: np.ndarray
    perm: np.ndarray       # tree order: perm[t] = original point id at tree position t
    leaf_lids_offset: np.ndarray  # nleaf+1 starts of each leaf in tree order
    skels: List[np.ndarray] = dataclasses.field(default_factory=list, repr=False)

    # ---- sizes the generated HGEMM bakes in ----
    @property
    def nrow(self) -> int:
        return len(self.nblockset) - 1

    @property
    def frow(self) -> int:
        return len(self.fblockset) - 1

    @property
    def cdepth(self) -> int:
        return len(self.clevelset) - 1

    @property
    def ncount(self) -> int:
        return len(self.npairx)

    @property
    def fcount(self) -> int:
        return len(self.fpairx)

    def offsets(self, nrhs: int):
        """(wptr, uptr, wskeloffset, uskeloffset, skel_total) for ``nrhs`` columns
        (``hcds.h:699-716`` and ``hcds.h:637-696``)."""
        wptr = (np.concatenate([[0], np.cumsum(self.Ddim[:-1].astype(np.int64))]) * nrhs)
        if wptr.size and wptr[-1] + int(self.Ddim[-1]) * nrhs > np.iinfo(np.int32).max:
            raise ValueError("leaf offsets overflow int32 for this nrhs")
        wsk = np.zeros(self.numnodes, np.int64)
        off = 0
        for v in self.cidx.tolist():
            wsk[v] = off
            off += int(self.slen[v]) * nrhs
        if off > np.iinfo(np.int32).max:
            raise ValueError("skeleton offsets overflow int32 for this nrhs")
        w32 = wptr.astype(np.int32)
        s32 = wsk.astype(np.int32)
        return w32, w32.copy(), s32, s32.copy(), off

    def flops(self, nrhs: int) -> int:
        """Algorithmic flops of one evaluation, ``compression.h:1079-1130``."""
        f = 0
        for v in range(1, self.numnodes):
            s = int(self.slen[v])
            if self.lchildren[v] == -1:
                f += 2 * s * nrhs * int(self.Ddim[self.lm[v]])
            else:
                f += 2 * s * (int(self.slen[self.lchildren[v]]) + int(self.slen[self.rchildren[v]])) * nrhs
        f *= 2
        dd = self.Ddim.astype(np.int64)
        f += int((2 * dd[self.npairx] * dd[self.npairy] * nrhs).sum())
        sl = self.slen.astype(np.int64)
        f += int((2 * sl[self.fpairx] * sl[self.fpairy] * nrhs).sum())
        return f

    def flops_breakdown(self, nrhs: int) -> Dict[str, int]:
        """Algorithmic flops per pass: tree (up + down projections), near, far."""
        tree = 0
        for v in range(1, self.numnodes):
            s = int(self.slen[v])
            if self.lchildren[v] == -1:
                tree += 2 * s * nrhs * int(self.Ddim[self.lm[v]])
            else:
                tree += 2 * s * (int(self.slen[self.lchildren[v]]) + int(self.slen[self.rchildren[v]])) * nrhs
        dd = self.Ddim.astype(np.int64)
        sl = self.slen.astype(np.int64)
        return {"tree": 2 * tree,
                "near": int((2 * dd[self.npairx] * dd[self.npairy] * nrhs).sum()),
                "far": int((2 * sl[self.fpairx] * sl[self.fpairy] * nrhs).sum())}

    def to_tree_order(self, W: np.ndarray) -> np.ndarray:
        """``transform`` (``hcds.h:766-788``): W (N x r, column-major) -> TW with each
        leaf's rows contiguous per column block (leaf-blocked, tree order)."""
        W = np.asarray(W)
        n, r = W.shape
        out = np.empty(n * r, dtype=W.dtype)
        for i in range(self.nleaf):
            a, b = int(self.leaf_lids_offset[i]), int(self.leaf_lids_offset[i + 1])
            rows = self.perm[a:b]
            blk = W[rows, :]
            out[a * r:b * r] = blk.reshape(-1, order="F")
        return out

    def from_tree_order(self, TY: np.ndarray, r: int) -> np.ndarray:
        """Inverse of :meth:`to_tree_order`: leaf-blocked result -> N x r original order."""
        Y = np.empty((self.n, r), dtype=TY.dtype)
        for i in range(self.nleaf):
            a, b = int(self.leaf_lids_offset[i]), int(self.leaf_lids_offset[i + 1])
            Y[self.perm[a:b], :] = TY[a * r:b * r].reshape(b - a, r, order="F")
        return Y

    # ---- persistence: raw little-endian arrays in one .npz ----
    _ARRAYS = ("D", "Dptr", "B", "Bptr", "VT", "VTptr", "lchildren", "rchildren", "levelset",
               "idx", "Ddim", "lm", "slen", "nblockset", "nblocks", "npairx", "npairy",
               "fblockset", "fblocks", "fpairx", "fpairy", "wpart", "clevelset", "cidx",
               "perm", "leaf_lids_offset")

    def save(self, path: str) -> None:
        meta = np.array([self.n, self.nleaf, self.numnodes, self.depth, int(self.is_hss)], np.int64)
        np.savez(path, meta=meta, **{k: getattr(self, k) for k in self._ARRAYS})

    @classmethod
    def load(cls, path: str) -> "CDS":
        z = np.load(path)
        n, nleaf, numnodes, depth, hss = (int(v) for v in z["meta"])
        return cls(n=n, nleaf=nleaf, numnodes=numnodes, depth=depth, is_hss=bool(hss),
                   **{k: z[k] for k in cls._ARRAYS})


# ---------------------------------------------------------------------------
# compression driver
# ---------------------------------------------------------------------------

def _workers() -> int:
    return max(1, min(32, os.cpu_count() or 1))


@contextlib.contextmanager
def _blas_single_thread():
    try:
        from threadpoolctl import threadpool_limits
    except Exception:  # pragma: no cover
        yield
        return
    with threadpool_limits(limits=1, user_api="blas"):
        yield

def _sample_rows(own: np.ndarray, cand: np.ndarray, nsamples: int, n: int,
                 rng: np.random.Generator) -> np.ndarray:
    """Rows for the ID of a node: nearest outside candidates first (up to half of
    ``nsamples``), then uniform random outside points (``compression.h:597-690``)."""
    if nsamples >= n - len(own):
        return np.arange(n, dtype=np.int64)
    taken = np.zeros(n, bool)
    taken[own] = True
    c = cand[~taken[cand]]
    _, first = np.unique(c, return_index=True)
    c = c[np.sort(first)][: nsamples // 2]
    taken[c] = True
    parts = [c]
    need = nsamples - len(c)
    while need > 0:
        draw = rng.integers(0, n, size=2 * need + 16)
        draw = draw[~taken[draw]]
        _, first = np.unique(draw, return_index=True)
        draw = draw[np.sort(first)][:need]
        taken[draw] = True
        parts.append(draw)
        need -= len(draw)
    return np.concatenate(parts).astype(np.int64)


# ---------------------------------------------------------------------------
# k-NN sampling of ID rows (matroxTest-V1/compression.h:362-443, 597-797)
# ---------------------------------------------------------------------------

KNN = 32  # neighbours per point (sympiler/HTree.cpp:35, `setup.k = 32`)


def _pair_gt(ad, ai, bd, bi):
    """(distance, id) pairs compared lexicographically, as std::pair<double, int> compares."""
    return (ad > bd) | ((ad == bd) & (ai > bi))


def _max_heap_rows(d: np.ndarray, ids: np.ndarray) -> None:
    """Arrange every row as a binary max-heap of (distance, id) pairs, in place.

    The reference keeps each point's neighbour list as the max-heap of its search
    (``sympiler/NearSearch.cpp:20-66`` leaves the lists unsorted), and its sampling reads the
    first and second halves of that array (``compression.h:372-391``).  Exact lists built
    here are given the same heap shape by a bottom-up heapify (Floyd's method)."""
    n, k = d.shape
    rows = np.arange(n)
    for start in range(k // 2 - 1, -1, -1):
        pos = np.full(n, start)
        live = rows
        while live.size:
            p = pos[live]
            c = 2 * p + 1
            ok = c < k
            live, p, c = live[ok], p[ok], c[ok]
            if not live.size:
                break
            c2 = c + 1
            has2 = c2 < k
            c2s = np.where(has2, c2, c)
            right = has2 & _pair_gt(d[live, c2s], ids[live, c2s], d[live, c], ids[live, c])
            c = np.where(right, c2s, c)
            swap = _pair_gt(d[live, c], ids[live, c], d[live, p], ids[live, p])
            live, p, c = live[swap], p[swap], c[swap]
            d[live, p], d[live, c] = d[live, c], d[live, p].copy()
            ids[live, p], ids[live, c] = ids[live, c], ids[live, p].copy()
            pos[live] = c


def knn_lists(X: np.ndarray, k: int = KNN, chunk: int = 2048) -> Tuple[np.ndarray, np.ndarray]:
    """Exact k nearest neighbours of every point (itself included) by squared Euclidean
    distance: (ids, distances), each N x k, every row laid out as a max-heap like the
    reference's lists.  Blocked distance products with torch (the GPU when one is present)."""
    import torch
    X = np.ascontiguousarray(X, dtype=np.float64)
    n = X.shape[0]
    k = min(k, n)
    dev = torch.device("cuda") if torch.cuda.is_available() else torch.device("cpu")
    T = torch.as_tensor(X, device=dev)
    sq = (T * T).sum(1)
    ids = np.empty((n, k), np.int64)
    dist = np.empty((n, k), np.float64)
    for a in range(0, n, chunk):
        b = min(n, a + chunk)
        d2 = (sq[a:b, None] + sq[None, :] - 2.0 * (T[a:b] @ T.T)).clamp_min_(0.0)
        d2[torch.arange(b - a, device=dev), torch.arange(a, b, device=dev)] = 0.0
        val, idx = torch.topk(d2, k, dim=1, largest=False, sorted=True)
        ids[a:b] = idx.cpu().numpy()
        dist[a:b] = val.cpu().numpy()
    # exact distances of the chosen pairs (the product form rounds), then ascending order
    dist = ((X[ids] - X[:, None, :]) ** 2).sum(2)
    order = np.lexsort((ids, dist), axis=1)
    ids = np.take_along_axis(ids, order, 1)
    dist = np.take_along_axis(dist, order, 1)
    _max_heap_rows(dist, ids)
    return ids, dist


def _leaf_neighbours(NN, DN, own, nsamples):
    """``BuildNeighBorsLeaf`` (compression.h:362-403): sampling neighbours of a leaf, in
    (distance, id) order, and its pruning set.  The first half of each point's list is the
    pruning set; the second half, sorted, gives the sampling neighbours outside both."""
    k = NN.shape[1]
    prune = np.setdiff1d(NN[own, :k // 2].ravel(), own)
    tid = NN[own, (k + 1) // 2:].T.ravel()
    tds = DN[own, (k + 1) // 2:].T.ravel()
    order = np.lexsort((tid, tds))[: (k - 1) * len(own) // 2]
    tid, tds = tid[order], tds[order]
    keep = ~np.isin(tid, prune) & ~np.isin(tid, own)
    tid, tds = tid[keep], tds[keep]
    _, first = np.unique(tid, return_index=True)
    first = np.sort(first)[:nsamples]
    return tid[first], tds[first]


def _internal_neighbours(lids, lds, rids, rds, own, lprune, rprune):
    """``BuildNeighBorsInternal`` (compression.h:405-443): the children's sampling neighbours
    merged (smallest distance per point), minus the node's points and the children's pruning
    sets, in (distance, id) order."""
    ids = np.concatenate([lids, rids])
    ds = np.concatenate([lds, rds])
    order = np.lexsort((ids, ds))
    ids, ds = ids[order], ds[order]
    _, first = np.unique(ids, return_index=True)
    first = np.sort(first)
    ids, ds = ids[first], ds[first]
    keep = ~np.isin(ids, own) & ~np.isin(ids, lprune) & ~np.isin(ids, rprune)
    return ids[keep], ds[keep]


def _fill_random(amap: np.ndarray, own: np.ndarray, nsamples: int, n: int,
                 rng: np.random.Generator) -> np.ndarray:
    """The reference's sample rows (compression.h:622-650, 720-755): the neighbour rows
    first, then uniform random points outside the node until ``nsamples``; every point when
    ``nsamples`` reaches the number of outside points."""
    if nsamples >= n - len(own):
        return np.arange(n, dtype=np.int64)
    taken = np.zeros(n, bool)
    taken[own] = True
    taken[amap] = True
    parts = [np.asarray(amap, np.int64)]
    need = nsamples - len(amap)
    while need > 0:
        draw = rng.integers(0, n, size=2 * need + 16)
        draw = draw[~taken[draw]]
        _, first = np.unique(draw, return_index=True)
        draw = draw[np.sort(first)][:need]
        taken[draw] = True
        parts.append(draw)
        need -= len(draw)
    return np.concatenate(parts).astype(np.int64)


def _fill_sequential(amap: np.ndarray, own: np.ndarray, nsamples: int, n: int, draw) -> np.ndarray:
    """As :func:`_fill_random`, but one draw at a time from ``draw()`` (a source of the
    values the reference's rand() returns), each accepted when it is neither a sample yet nor
    a point of the node (compression.h:640-648)."""
    if nsamples >= n - len(own):
        return np.arange(n, dtype=np.int64)
    out = [int(v) for v in amap]
    taken = set(out)
    taken.update(int(v) for v in own)
    while len(out) < nsamples:
        sample = draw() % n
        if sample not in taken:
            taken.add(sample)
            out.append(sample)
    return np.asarray(out, dtype=np.int64)


def build_cds(X: np.ndarray, kernel: KernelSpec, leaf_size: int = 256, budget: float = 0.03,
              tol: float = 1e-5, max_rank: int = 256, seed: int = 0,
              neighbour_leaves: int = 4, id_on_gpu: bool = False, structure=None,
              sampling: str = "knn", rand_source=None) -> CDS:
    """Build the CDS of the kernel matrix of point set X (N x d, row-major).

    ``id_on_gpu``: the sample matrices of each tree level are computed on the GPU
    (``mxb_kernel_blocks``) and factored there in one launch (``mxb_batched_id``) instead of
    one host ID per node; sampling and the tree stay on the host.

    ``structure``: a :class:`~matrox_ru_b200.structure_bin.Structure` (tree, near and far
    lists), e.g. read from the reference's ``.bin`` files, used instead of building one;
    ``budget`` is then unused and ``leaf_size`` only sizes the samples.

    ``sampling``: how the ID picks kernel rows outside a node.  "knn" (default) is the
    reference's scheme (``compression.h:362-443, 597-797``) on 32-NN lists: the structure's
    own lists when it carries them (the reference generator's ``NN.bin``), else exact lists
    from :func:`knn_lists`.  "leaves" takes nearest outside points of the
    ``neighbour_leaves`` closest leaves instead (no neighbour search).

    ``rand_source``: a callable returning the successive values of the reference's rand()
    (k-NN sampling only).  The random sample rows of every node are then drawn from it one
    at a time, nodes in the reference's order (leaves, then each level upwards, node ids
    ascending), so a single-threaded reference run is reproduced draw for draw; by default
    each node draws from its own seeded generator."""
    if sampling not in ("knn", "leaves"):
        raise ValueError(f"sampling must be 'knn' or 'leaves', not {sampling!r}")
    X = np.ascontiguousarray(X, dtype=np.float64)
    n = X.shape[0]
    if structure is None:
        tree = build_tree(X, leaf_size)
        near = near_lists(tree, budget)
        far = far_lists(tree, near)
    else:
        tree, near, far = structure.tree, structure.near, structure.far
        if sum(len(tree.lids[tree.leaf_node(i)]) for i in range(tree.nleaf)) != n:
            raise ValueError("the structure's leaves do not hold the N points of X")
    is_hss = all(len(l) == 1 for l in near)
    nn = tree.numnodes

    lch = np.full(nn, -1, np.int32)
    rch = np.full(nn, -1, np.int32)
    for v in range(tree.first_leaf):
        lch[v], rch[v] = 2 * v + 1, 2 * v + 2
    lm = np.full(nn, -1, np.int32)
    for i in range(tree.nleaf):
        lm[tree.leaf_node(i)] = i
    Ddim = np.array([len(tree.lids[tree.leaf_node(i)]) for i in range(tree.nleaf)], np.int32)

    # neighbour candidates per leaf: outside points of the closest leaves, by distance
    cand: List[np.ndarray] = [np.zeros(0, np.int64)] * nn
    # k-NN sampling state per node: sampling neighbours (ids, distances) and pruning set
    NN = DN = None
    snb: List[Tuple[np.ndarray, np.ndarray]] = [(np.zeros(0, np.int64), np.zeros(0))] * nn
    prune: List[np.ndarray] = [np.zeros(0, np.int64)] * nn
    if sampling == "knn":
        if structure is not None and structure.NN is not None and structure.distNN is not None \
                and structure.NN.size == structure.distNN.size and structure.NN.size % n == 0:
            k = structure.NN.size // n
            NN = np.asarray(structure.NN, np.int64).reshape(n, k)
            DN = np.asarray(structure.distNN, np.float64).reshape(n, k)
        else:
            NN, DN = knn_lists(X, KNN)
    elif tree.nleaf > 1:
        dm = np.sqrt(sqdist(tree.mid, tree.mid))
        for i in range(tree.nleaf):
            order = [j for j in np.argsort(dm[i], kind="stable") if j != i][:neighbour_leaves]
            own = tree.lids[tree.leaf_node(i)]
            pool = np.concatenate([tree.lids[tree.leaf_node(j)] for j in order])
            dist = sqdist(X[pool], X[own]).min(1)
            cand[tree.leaf_node(i)] = pool[np.argsort(dist, kind="stable")]

    slen = np.zeros(nn, np.int32)
    skels: List[np.ndarray] = [np.zeros(0, np.int64)] * nn
    proj: List[np.ndarray] = [np.zeros((0, 0))] * nn

    def prepare_knn(v: int):
        own = np.asarray(tree.lids[v], np.int64)
        if lch[v] == -1:
            bmap = own
            nsamples = max(2 * len(bmap), 2 * leaf_size)
            ids, ds = _leaf_neighbours(NN, DN, own, nsamples)
            amap0 = ids
        else:
            l, r = int(lch[v]), int(rch[v])
            bmap = np.concatenate([skels[l], skels[r]])
            nsamples = max(2 * len(bmap), 2 * leaf_size)
            ids, ds = _internal_neighbours(snb[l][0], snb[l][1], snb[r][0], snb[r][1], own, prune[l], prune[r])
            amap0 = ids[:nsamples]
        if rand_source is not None:
            amap = _fill_sequential(amap0, own, nsamples, n, rand_source)
        else:
            amap = _fill_random(amap0, own, nsamples, n, np.random.default_rng([seed, v]))
        return v, amap, bmap, (ids, ds)

    def prepare(v: int):
        if NN is not None:
            return prepare_knn(v)
        own = tree.lids[v]
        if lch[v] == -1:
            bmap = own
            cv = cand[v]
            keep = None
        else:
            l, r = int(lch[v]), int(rch[v])
            bmap = np.concatenate([skels[l], skels[r]])
            merged = np.concatenate([cand[l], cand[r]])
            owns = np.zeros(n, bool)
            owns[own] = True
            merged = merged[~owns[merged]]
            if merged.size:
                dist = sqdist(X[merged], X[bmap]).min(1)
                merged = merged[np.argsort(dist, kind="stable")]
                _, first = np.unique(merged, return_index=True)
                merged = merged[np.sort(first)]
            cv = merged
            keep = merged[: 4 * leaf_size]
        nsamples = max(2 * len(bmap), 2 * leaf_size)
        amap = _sample_rows(own, cv, nsamples, n, np.random.default_rng([seed, v]))
        return v, amap, bmap, keep

    def compress_prepared(prep):
        v, amap, bmap, keep = prep
        K = kernel_matrix(X, amap, bmap, kernel)
        piv, P = interpolative_decomposition(np.asfortranarray(K), tol, max_rank)
        return v, bmap[piv], P, keep

    def compress(v: int):
        return compress_prepared(prepare(v))

    def prepare_level(pool, nodes):
        # one shared draw sequence: sample the level's nodes one after the other, in order
        return [prepare(v) for v in nodes] if rand_source is not None else list(pool.map(prepare, nodes))

    def compress_level_on_gpu(pool, nodes):
        from . import hgemm as H
        prep = prepare_level(pool, nodes)
        K, _ = H.kernel_matrices(dX, kernel, [q[1] for q in prep], [q[2] for q in prep])
        ids = H.batched_id(K, [(len(q[1]), len(q[2])) for q in prep], tol, max_rank)
        del K
        return [(v, bmap[piv], P, keep) for (v, _, bmap, keep), (piv, P) in zip(prep, ids)]

    dX = None
    if id_on_gpu:
        import torch
        dX = torch.as_tensor(X).to("cuda")
    # nodes of one level are independent: LAPACK / BLAS release the GIL, so a thread pool
    # over the level with single-threaded BLAS inside scales with the host cores
    with _blas_single_thread(), ThreadPoolExecutor(max_workers=_workers()) as pool:
        for lev in range(tree.depth, 0, -1):
            nodes = list(range((1 << lev) - 1, (1 << (lev + 1)) - 1))
            if id_on_gpu:
                level = compress_level_on_gpu(pool, nodes)
            elif rand_source is not None and NN is not None:
                level = pool.map(compress_prepared, prepare_level(pool, nodes))
            else:
                level = pool.map(compress, nodes)
            for v, sk, P, keep in level:
                skels[v] = sk
                proj[v] = P
                slen[v] = P.shape[0]
                if NN is not None:
                    # the node's pruning set becomes its skeleton points' first half-lists
                    # (compression.h:682-687, 783-788)
                    snb[v] = keep
                    prune[v] = np.unique(NN[np.asarray(sk, np.int64), :NN.shape[1] // 2].ravel())
                elif keep is not None:
                    cand[v] = keep

    # ---- pack (hcds.h) ----
    levelset, idx = levelsets_top_down(tree)
    clevelset, wpart, cidx = coarsened_levels(tree)

    VTptr = np.zeros(nn, np.int32)
    off = 0
    for v in cidx.tolist():
        VTptr[v] = off
        off += proj[v].size
    if off > np.iinfo(np.int32).max:
        raise ValueError("projection storage overflows int32 offsets")
    VT = np.empty(off)
    for v in cidx.tolist():
        VT[VTptr[v]:VTptr[v] + proj[v].size] = proj[v].reshape(-1, order="F")

    if is_hss:
        npx = np.arange(tree.nleaf, dtype=np.int32)
        npy = npx.copy()
        nblockset = np.array([0], np.int32)
        nblocks = np.array([0], np.int32)
        fpx = np.arange(1, nn, dtype=np.int32)
        fpy = np.array([v - 1 if v % 2 == 0 else v + 1 for v in range(1, nn)], np.int32)
        fblockset = np.array([0], np.int32)
        fblocks = np.array([0], np.int32)
        for v in range(1, nn):
            assert far[v] == [int(fpy[v - 1])], "HSS far lists must be siblings"
    else:
        nblockset, nblocks, npx, npy = blocked_near(tree, near)
        fblockset, fblocks, fpx, fpy = blocked_far(tree, far)

    Dsz = Ddim.astype(np.int64)[npx] * Ddim.astype(np.int64)[npy]
    Dptr = np.concatenate([[0], np.cumsum(Dsz)[:-1]]).astype(np.uint64)
    D = np.empty(int(Dsz.sum()))

    def near_block(k):
        x, y = int(npx[k]), int(npy[k])
        blk = kernel_matrix(X, tree.lids[tree.leaf_node(x)], tree.lids[tree.leaf_node(y)], kernel)
        D[int(Dptr[k]):int(Dptr[k]) + blk.size] = blk.reshape(-1, order="F")

    Bsz = slen.astype(np.int64)[fpx] * slen.astype(np.int64)[fpy]
    Bptr = (np.concatenate([[0], np.cumsum(Bsz)[:-1]]) if len(fpx) else np.zeros(0)).astype(np.uint64)
    B = np.empty(int(Bsz.sum()))

    def far_block(k):
        x, y = int(fpx[k]), int(fpy[k])
        blk = kernel_matrix(X, skels[x], skels[y], kernel)
        B[int(Bptr[k]):int(Bptr[k]) + blk.size] = blk.reshape(-1, order="F")

    with _blas_single_thread(), ThreadPoolExecutor(max_workers=_workers()) as pool:
        list(pool.map(near_block, range(len(npx))))
        list(pool.map(far_block, range(len(fpx))))

    perm = np.concatenate([tree.lids[tree.leaf_node(i)] for i in range(tree.nleaf)]).astype(np.int64)
    lofs = np.concatenate([[0], np.cumsum(Ddim.astype(np.int64))]).astype(np.int64)

    return CDS(n=n, nleaf=tree.nleaf, numnodes=nn, depth=tree.depth, is_hss=is_hss,
               D=D, Dptr=Dptr, B=B, Bptr=Bptr, VT=VT, VTptr=VTptr, lchildren=lch, rchildren=rch,
               levelset=levelset, idx=idx, Ddim=Ddim, lm=lm, slen=slen,
               nblockset=nblockset, nblocks=nblocks, npairx=npx, npairy=npy,
               fblockset=fblockset, fblocks=fblocks, fpairx=fpx, fpairy=fpy,
               wpart=wpart, clevelset=clevelset, cidx=cidx, perm=perm,
               leaf_lids_offset=lofs, skels=skels)


def dense_kernel_times(X: np.ndarray, W: np.ndarray, kernel: KernelSpec, rows=None,
                       chunk: int = 4096) -> np.ndarray:
    """Dense FP64 K(X[rows], X) @ W, chunked over columns of K (the dense oracle)."""
    X = np.ascontiguousarray(X, dtype=np.float64)
    n = X.shape[0]
    rows = np.arange(n) if rows is None else np.asarray(rows)
    out = np.zeros((len(rows), W.shape[1]))
    for a in range(0, n, chunk):
        b = min(n, a + chunk)
        out += kernel_matrix(X, rows, np.arange(a, b), kernel) @ W[a:b]
    return out
