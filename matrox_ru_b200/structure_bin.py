"""The reference's on-disk structure format: the ``.bin`` files that the Sympiler generator
writes (``HTree::savetree2disk``, ``sympiler/HTree.cpp:468-542``, with the arrays built in
``sympiler/HTree.cpp:398-456``) and that the MatRox driver reads back (``readHtree``,
``matroxTest-V1/HTree.h:76-243``).

One file per array, raw little-endian int32 (``distNN.bin``: float64), no header: every
length is implied by the file size, as ``preprocesoffset`` (``matroxTest-V1/Util.h:41-47``)
reads it.

* :func:`write_structure` exports a :class:`Structure` (tree, near lists, far lists) in that
  layout, so the reference's driver can run on a structure built here.
* :func:`read_structure` imports one, so a structure written by the Sympiler generator can be
  compressed here (``structure.build_cds(..., structure=...)``) and evaluated on the GPU.
  The tree must be a perfect binary tree in heap numbering (children of v at 2v+1 and 2v+2,
  leaves last), the layout the reference's evaluators assume.
"""
from __future__ import annotations

import dataclasses
import os
from typing import Dict, List, Optional

import numpy as np

from . import structure as S

# file name -> what it holds (matroxTest-V1/HTree.h:76-243 reads them in this order)
FILES = {
    "NN.bin": "k nearest neighbours of every point, int32 (may be empty)",
    "distNN.bin": "their distances, float64, one per NN.bin entry",
    "clevelset.bin": "coarsened level sets: cdepth + 1 offsets into wpart",
    "cidx.bin": "nodes of the coarsened partitions, numnodes - 1 entries",
    "wpart.bin": "partition offsets into cidx",
    "levelset.bin": "level sets from the root's children down: depth + 1 offsets into idx",
    "idx.bin": "nodes of the level sets, numnodes - 1 entries",
    "nblockset.bin": "near blocking: block-row offsets into nblocks (H2-b only)",
    "nblocks.bin": "near blocking: block offsets into nxval / nyval (H2-b only)",
    "nxval.bin": "near pairs: leaf index of the output block",
    "nyval.bin": "near pairs: leaf index of the input block",
    "fblockset.bin": "far blocking: block-row offsets into fblocks (H2-b only)",
    "fblocks.bin": "far blocking: block offsets into fxval / fyval (H2-b only)",
    "fxval.bin": "far pairs: node of the output skeleton",
    "fyval.bin": "far pairs: node of the input skeleton",
    "dim.bin": "points per leaf (nleaf entries)",
    "leafmap.bin": "leaf index of every node, -1 for internal nodes (numnodes entries)",
    "lids.bin": "point ids of every node except the root, node after node",
    "lidsoffset.bin": "offset of every node's ids in lids (numnodes entries; root 0)",
    "lidslen.bin": "number of ids of every node (numnodes entries; root 0)",
    "lchildren.bin": "left child of every node, -1 for leaves",
    "rchildren.bin": "right child of every node, -1 for leaves",
}
BLOCK_FILES = ("nblockset.bin", "nblocks.bin", "fblockset.bin", "fblocks.bin")


@dataclasses.dataclass
class Structure:
    """A cluster tree with its near lists (per leaf, leaf indices) and far lists (per node,
    node ids), the input of the compression."""
    tree: S.Tree
    near: List[List[int]]
    far: List[List[int]]
    NN: Optional[np.ndarray] = None      # flattened k-NN lists, when known
    distNN: Optional[np.ndarray] = None

    @property
    def is_hss(self) -> bool:
        return all(len(lst) == 1 for lst in self.near)


def build_structure(X: np.ndarray, leaf_size: int = 256, budget: float = 0.03) -> Structure:
    """The tree and interaction lists that ``structure.build_cds`` builds for X."""
    X = np.ascontiguousarray(X, dtype=np.float64)
    tree = S.build_tree(X, leaf_size)
    near = S.near_lists(tree, budget)
    return Structure(tree, near, S.far_lists(tree, near))


def structure_arrays(st: Structure) -> Dict[str, np.ndarray]:
    """Every file's array, in the reference's layout."""
    tree = st.tree
    nn, nl = tree.numnodes, tree.nleaf
    i32 = np.int32
    lch = np.full(nn, -1, i32)
    rch = np.full(nn, -1, i32)
    for v in range(tree.first_leaf):
        lch[v], rch[v] = 2 * v + 1, 2 * v + 2
    lm = np.full(nn, -1, i32)
    for i in range(nl):
        lm[tree.leaf_node(i)] = i
    dim = np.array([len(tree.lids[tree.leaf_node(i)]) for i in range(nl)], i32)
    levelset, idx = S.levelsets_top_down(tree)
    clevelset, wpart, cidx = S.coarsened_levels(tree)
    out = {"clevelset.bin": clevelset, "cidx.bin": cidx, "wpart.bin": wpart, "levelset.bin": levelset,
           "idx.bin": idx, "dim.bin": dim, "leafmap.bin": lm, "lchildren.bin": lch, "rchildren.bin": rch}
    if st.is_hss:
        out["nxval.bin"] = np.arange(nl, dtype=i32)
        out["nyval.bin"] = np.arange(nl, dtype=i32)
        out["fxval.bin"] = np.arange(1, nn, dtype=i32)
        out["fyval.bin"] = np.array([v - 1 if v % 2 == 0 else v + 1 for v in range(1, nn)], i32)
    else:
        out["nblockset.bin"], out["nblocks.bin"], out["nxval.bin"], out["nyval.bin"] = S.blocked_near(tree, st.near)
        out["fblockset.bin"], out["fblocks.bin"], out["fxval.bin"], out["fyval.bin"] = S.blocked_far(tree, st.far)
    # point ids node after node, level by level from the leaves up, root excluded
    # (sympiler/HTree.cpp:431-456)
    lofs = np.zeros(nn, i32)
    llen = np.zeros(nn, i32)
    parts = []
    off = 0
    for v in S.node_order_bottom_up(tree):
        lofs[v] = off
        llen[v] = len(tree.lids[v])
        parts.append(np.asarray(tree.lids[v], dtype=i32))
        off += len(tree.lids[v])
    out["lids.bin"] = np.concatenate(parts) if parts else np.zeros(0, i32)
    out["lidsoffset.bin"] = lofs
    out["lidslen.bin"] = llen
    out["NN.bin"] = np.asarray(st.NN if st.NN is not None else np.zeros(0), dtype=i32)
    out["distNN.bin"] = np.asarray(st.distNN if st.distNN is not None else np.zeros(0), dtype=np.float64)
    return out


def write_structure(st: Structure, directory: str) -> List[str]:
    """Write the structure's files into ``directory`` (created if needed); returns their names."""
    os.makedirs(directory, exist_ok=True)
    arrays = structure_arrays(st)
    for name, a in arrays.items():
        dt = "<f8" if name == "distNN.bin" else "<i4"
        np.ascontiguousarray(a).astype(dt).tofile(os.path.join(directory, name))
    return sorted(arrays)


def _read(directory: str, name: str, required: bool = True) -> Optional[np.ndarray]:
    path = os.path.join(directory, name)
    if not os.path.exists(path):
        if required:
            raise FileNotFoundError(f"{path}: missing structure file")
        return None
    size = os.path.getsize(path)
    item = 8 if name == "distNN.bin" else 4
    if size % item:
        raise ValueError(f"{path}: size {size} is not a multiple of {item} bytes")
    return np.fromfile(path, dtype="<f8" if item == 8 else "<i4").astype(np.float64 if item == 8 else np.int64)


def read_structure(directory: str, X: np.ndarray) -> Structure:
    """Read a structure written by :func:`write_structure` or by the Sympiler generator.
    X (N x d) supplies the leaf bounding boxes used to pick sampling candidates."""
    X = np.ascontiguousarray(X, dtype=np.float64)
    dim = _read(directory, "dim.bin")
    nl = len(dim)
    if nl < 1 or nl & (nl - 1):
        raise ValueError(f"dim.bin: {nl} leaves; a perfect binary tree needs a power of two")
    nn = 2 * nl - 1
    depth = nl.bit_length() - 1
    first = nl - 1
    lch, rch, lm = _read(directory, "lchildren.bin"), _read(directory, "rchildren.bin"), _read(directory, "leafmap.bin")
    lofs, llen, lids = _read(directory, "lidsoffset.bin"), _read(directory, "lidslen.bin"), _read(directory, "lids.bin")
    for name, a in (("lchildren.bin", lch), ("rchildren.bin", rch), ("leafmap.bin", lm), ("lidsoffset.bin", lofs),
                    ("lidslen.bin", llen)):
        if len(a) != nn:
            raise ValueError(f"{name}: {len(a)} entries, expected {nn}")
    for v in range(nn):
        leaf = v >= first
        want = (-1, -1, v - first) if leaf else (2 * v + 1, 2 * v + 2, -1)
        if (lch[v], rch[v], lm[v]) != want:
            raise ValueError(f"node {v}: the tree is not a perfect binary tree in heap numbering")
    n = X.shape[0]
    node_ids: List[Optional[np.ndarray]] = [None] * nn
    for v in range(1, nn):
        a, ln = int(lofs[v]), int(llen[v])
        if a < 0 or ln < 0 or a + ln > len(lids):
            raise ValueError(f"node {v}: ids [{a}, {a + ln}) outside lids.bin")
        ids = lids[a:a + ln]
        if ids.size and (ids.min() < 0 or ids.max() >= n):
            raise ValueError(f"node {v}: point id outside the {n} points")
        node_ids[v] = ids
    if nl == 1:
        node_ids[0] = np.arange(n, dtype=np.int64)
    else:
        node_ids[0] = np.concatenate([node_ids[1], node_ids[2]])
    for i in range(nl):
        if len(node_ids[first + i]) != dim[i]:
            raise ValueError(f"leaf {i}: {len(node_ids[first + i])} ids, dim.bin says {dim[i]}")
    for v in range(first):
        kids = np.concatenate([node_ids[2 * v + 1], node_ids[2 * v + 2]])
        if v > 0 and not np.array_equal(np.sort(kids), np.sort(node_ids[v])):
            raise ValueError(f"node {v}: its ids are not the union of its children's")
    if not np.array_equal(np.sort(node_ids[0]), np.arange(n)):
        raise ValueError("the leaves do not partition the points")
    mids = np.empty((nl, X.shape[1]))
    rads = np.empty(nl)
    for i in range(nl):
        P = X[node_ids[first + i]]
        lo, hi = P.min(0), P.max(0)
        mids[i] = 0.5 * (lo + hi)
        rads[i] = np.sqrt(((hi - mids[i]) ** 2).sum())
    tree = S.Tree(depth, nn, nl, node_ids, mids, rads)
    nx, ny = _read(directory, "nxval.bin"), _read(directory, "nyval.bin")
    fx, fy = _read(directory, "fxval.bin"), _read(directory, "fyval.bin")
    if len(nx) != len(ny) or len(fx) != len(fy):
        raise ValueError("pair lists of unequal length")
    near: List[List[int]] = [[] for _ in range(nl)]
    for x, y in zip(nx.tolist(), ny.tolist()):
        if not (0 <= x < nl and 0 <= y < nl):
            raise ValueError(f"near pair ({x}, {y}) outside the {nl} leaves")
        near[x].append(y)
    far: List[List[int]] = [[] for _ in range(nn)]
    for x, y in zip(fx.tolist(), fy.tolist()):
        if not (0 < x < nn and 0 < y < nn):
            raise ValueError(f"far pair ({x}, {y}) outside the non-root nodes")
        far[x].append(y)
    NN = _read(directory, "NN.bin", required=False)
    dist = _read(directory, "distNN.bin", required=False)
    return Structure(tree, [sorted(v) for v in near], [sorted(v) for v in far],
                     None if NN is None or not NN.size else NN,
                     None if dist is None or not dist.size else dist)
