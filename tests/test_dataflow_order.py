"""CPU: the unit order of chained tree sweeps under per-node counters (the host scheduler of the
dataflow launches, through its test hook ``mxb_debug_dataflow_order``; no device needed).

The launches' waits end only if every unit's inputs come earlier in the claim order, and they are
counted right only if every counter index and unit count matches the producing nodes; both are
checked here on up-sweep trees (children before parents), down-sweep trees (parents before
children, leaf down after each leaf), ragged trees and forests of several plans.
"""
import ctypes

import numpy as np
import pytest

from matrox_ru_b200 import _lib, build


@pytest.fixture(scope="module")
def lib():
    build.build()
    return _lib.load()


def order(lib, deps, ntask, kt, ncol=3, workers=8):
    n = len(deps)
    first = np.zeros(n + 1, dtype=np.int32)
    first[1:] = np.cumsum([len(d) for d in deps])
    flat = np.array([x for d in deps for x in d] or [0], dtype=np.int32)
    ntask = np.asarray(ntask, dtype=np.int32)
    kt = np.asarray(kt, dtype=np.int32)
    cap = int(ntask.sum()) * ncol
    outs = [np.zeros(cap, dtype=np.int32) for _ in range(6)]
    count = ctypes.c_int64()
    ptr = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    rc = lib.mxb_debug_dataflow_order(n, ptr(first), ptr(flat), ptr(ntask), ptr(kt), ncol, workers,
                                      *[ptr(o) for o in outs], cap, ctypes.byref(count))
    if rc:
        return rc, None
    c = count.value
    node, col, dep0, dep1, need, sig = (o[:c] for o in outs)
    return rc, dict(node=node, col=col, dep0=dep0, dep1=dep1, need=need, sig=sig)


def up_tree(leaves, rows=2):
    """Heap-numbered binary up sweep: leaves read nothing, a parent reads its two children."""
    deps, ntask, kt = [], [], []
    ids = {}
    level = list(range(leaves))
    for i in level:
        ids[("leaf", i)] = len(deps)
        deps.append([])
        ntask.append(rows)
        kt.append(4)
    cur = [ids[("leaf", i)] for i in range(leaves)]
    while len(cur) > 2:
        nxt = []
        for a, b in zip(cur[0::2], cur[1::2]):
            nxt.append(len(deps))
            deps.append([a, b])
            ntask.append(rows)
            kt.append(8)
        cur = nxt
    return deps, ntask, kt


def down_tree(depth, rows=2):
    """Down sweep with leaf down: a node reads its parent; each leaf's leaf-down block reads the
    leaf's down node."""
    deps, ntask, kt = [[], []], [rows, rows], [4, 4]  # the two nodes below the root
    cur = [0, 1]
    for _ in range(depth):
        nxt = []
        for p in cur:
            for _ in range(2):
                nxt.append(len(deps))
                deps.append([p])
                ntask.append(rows)
                kt.append(4)
        cur = nxt
    for leaf in cur:
        deps.append([leaf])
        ntask.append(rows)
        kt.append(4)
    return deps, ntask, kt


def check_invariants(deps, ntask, out, ncol):
    node, col = out["node"], out["col"]
    n = len(deps)
    # every (node, column) unit of every row tile exactly once
    seen = {}
    for u, (x, c) in enumerate(zip(node, col)):
        seen.setdefault((int(x), int(c)), []).append(u)
    assert len(seen) == n * ncol
    assert all(len(v) == ntask[x] for (x, _), v in seen.items())
    # inputs first: every unit of a node's inputs, in the same column tile, comes earlier
    for (x, c), us in seen.items():
        for d in deps[x]:
            assert max(seen[(d, c)]) < min(us), (x, d, c)
    # counters: a producing node signals its own counter block, its readers wait on it with the
    # producer's row-tile count; nodes nobody reads signal nothing
    readers = {d for ds in deps for d in ds}
    sig_of = {}
    for u, x in enumerate(node):
        s = int(out["sig"][u])
        if x in readers:
            assert s >= 0
            sig_of.setdefault(int(x), set()).add(s - int(col[u]))
        else:
            assert s == -1
    assert all(len(v) == 1 for v in sig_of.values())
    base = {x: next(iter(v)) for x, v in sig_of.items()}
    blocks = sorted(base.values())
    assert all(b - a >= ncol for a, b in zip(blocks, blocks[1:]))  # disjoint counter blocks
    for u, x in enumerate(node):
        ds = deps[int(x)]
        got = [int(out["dep0"][u]), int(out["dep1"][u])]
        want = [base[d] + int(col[u]) for d in ds] + [-1] * (2 - len(ds))
        assert got == want
        need = int(out["need"][u])
        assert [need & 0xFFFF, need >> 16][:len(ds)] == [ntask[d] for d in ds]


@pytest.mark.parametrize("leaves,workers", [(2, 1), (16, 4), (64, 148), (256, 148)])
def test_up_sweep_order(lib, leaves, workers):
    deps, ntask, kt = up_tree(leaves)
    rc, out = order(lib, deps, ntask, kt, ncol=3, workers=workers)
    assert rc == 0
    check_invariants(deps, ntask, out, 3)


@pytest.mark.parametrize("depth,workers", [(0, 1), (3, 8), (6, 148)])
def test_down_sweep_order(lib, depth, workers):
    deps, ntask, kt = down_tree(depth)
    rc, out = order(lib, deps, ntask, kt, ncol=4, workers=workers)
    assert rc == 0
    check_invariants(deps, ntask, out, 4)


def test_parent_follows_its_children_closely(lib):
    """Depth-first priority: with many more units than workers, a parent's units come soon after
    its children's, long before the last leaves (so the children's tiles are still in L2)."""
    deps, ntask, kt = up_tree(256)
    rc, out = order(lib, deps, ntask, kt, ncol=8, workers=148)
    assert rc == 0
    node = out["node"]
    first_pos = {}
    for u, x in enumerate(node):
        first_pos.setdefault(int(x), u)
    parent01 = 256  # the first internal node reads leaves 0 and 1
    assert deps[parent01] == [0, 1]
    last_leaf_pos = max(first_pos[i] for i in range(256))
    assert first_pos[parent01] < last_leaf_pos / 4


def test_ragged_forest_of_two_plans(lib):
    """Two up-sweep trees of different shapes (row tiles 1-3, K tiles 1-9) in one launch."""
    d1, n1, k1 = up_tree(8, rows=3)
    d2, n2, k2 = up_tree(32, rows=1)
    off = len(d1)
    deps = d1 + [[x + off for x in d] for d in d2]
    rng = np.random.default_rng(3)
    ntask = [int(x) for x in rng.integers(1, 4, size=len(deps))]
    kt = [int(x) for x in rng.integers(1, 10, size=len(deps))]
    rc, out = order(lib, deps, ntask, kt, ncol=2, workers=5)
    assert rc == 0
    check_invariants(deps, ntask, out, 2)


def test_non_trees_are_refused(lib):
    # a node read by two nodes AND a node reading two nodes: neither an in-tree nor an out-tree
    deps = [[], [], [0, 1], [0], [2]]
    assert order(lib, deps, [1] * 5, [1] * 5)[0] == _lib.MXB_ERR_UNSUPPORTED
    # a cycle
    assert order(lib, [[1], [0]], [1, 1], [1, 1])[0] == _lib.MXB_ERR_UNSUPPORTED
    # three inputs
    assert order(lib, [[], [], [], [0, 1, 2]], [1] * 4, [1] * 4)[0] == _lib.MXB_ERR_UNSUPPORTED
