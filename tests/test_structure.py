"""CPU: invariants of the host CDS producer (reference layout, exact block partition)."""
import numpy as np
import pytest

from matrox_ru_b200 import structure as S


def covered(cds):
    """Count how often each (leaf_i, leaf_j) block is covered by near + far pairs."""
    nl = cds.nleaf
    cnt = np.zeros((nl, nl), np.int32)
    first = cds.numnodes - nl

    def leaves(v):
        lo, hi = v, v
        while lo < first:
            lo, hi = 2 * lo + 1, 2 * hi + 2
        return np.arange(lo - first, hi - first + 1)
    for x, y in zip(cds.npairx, cds.npairy):
        cnt[x, y] += 1
    for x, y in zip(cds.fpairx, cds.fpairy):
        cnt[np.ix_(leaves(x), leaves(y))] += 1
    return cnt


@pytest.mark.parametrize("name", ["hss", "h2b", "ragged"])
def test_blocks_partition_the_matrix(small_cases, name):
    """Every block of the N x N matrix is represented exactly once (near or far)."""
    cds = small_cases[name]
    assert (covered(cds) == 1).all()


def test_budget_rule_near_count():
    X = S.gaussian_mixture(2048, 3, 4, 0, 3, 0.4, None, seed=1)
    t = S.build_tree(X, 64)
    assert t.nleaf == 32
    for budget, want in [(0.0, 1), (0.1, 2), (0.25, 7)]:
        near = S.near_lists(t, budget)
        assert all(len(l) == max(1, min(want, int(32 * budget - 1))) for l in near), budget


def test_hss_far_pairs_are_siblings(small_cases):
    cds = small_cases["hss"]
    assert cds.is_hss
    for i, (x, y) in enumerate(zip(cds.fpairx, cds.fpairy)):
        assert x == i + 1 and y == (x - 1 if x % 2 == 0 else x + 1)


def test_schedules_cover_every_nonroot_node_once(small_cases):
    for cds in small_cases.values():
        assert sorted(cds.cidx.tolist()) == list(range(1, cds.numnodes))
        assert sorted(cds.idx.tolist()) == list(range(1, cds.numnodes))
        # post-order inside partitions: children precede parents within a coarse level
        pos = {v: i for i, v in enumerate(cds.cidx.tolist())}
        for v in range(1, cds.numnodes):
            if cds.lchildren[v] != -1:
                assert pos[cds.lchildren[v]] < pos[v] and pos[cds.rchildren[v]] < pos[v]


def test_blocked_lists_consistent(small_cases):
    cds = small_cases["h2b"]
    assert cds.nblocks[cds.nblockset[-1]] == cds.ncount
    assert cds.fblocks[cds.fblockset[-1]] == cds.fcount
    # near block rows of 2 leaves: every pair of row i has x // 2 == i
    for i in range(cds.nrow):
        for j in range(cds.nblockset[i], cds.nblockset[i + 1]):
            for k in range(cds.nblocks[j], cds.nblocks[j + 1]):
                assert cds.npairx[k] // 2 == i


def test_flops_formula(small_cases):
    cds = small_cases["h2b"]
    r = 7
    f = 0
    for v in range(1, cds.numnodes):
        s = int(cds.slen[v])
        if cds.lchildren[v] == -1:
            f += 2 * s * r * int(cds.Ddim[cds.lm[v]])
        else:
            f += 2 * s * (int(cds.slen[cds.lchildren[v]]) + int(cds.slen[cds.rchildren[v]])) * r
    f *= 2
    for x, y in zip(cds.npairx, cds.npairy):
        f += 2 * int(cds.Ddim[x]) * int(cds.Ddim[y]) * r
    for x, y in zip(cds.fpairx, cds.fpairy):
        f += 2 * int(cds.slen[x]) * int(cds.slen[y]) * r
    assert cds.flops(r) == f


def test_tree_order_roundtrip(small_cases):
    cds = small_cases["ragged"]
    W = np.random.default_rng(0).standard_normal((cds.n, 5))
    assert np.array_equal(cds.from_tree_order(cds.to_tree_order(W), 5), W)


def test_save_load_roundtrip(tmp_path, small_cases):
    cds = small_cases["h2b"]
    p = tmp_path / "c.npz"
    cds.save(str(p))
    back = S.CDS.load(str(p))
    for k in S.CDS._ARRAYS:
        assert np.array_equal(getattr(cds, k), getattr(back, k)), k
    assert (back.n, back.nleaf, back.numnodes, back.is_hss) == (cds.n, cds.nleaf, cds.numnodes, cds.is_hss)


def test_offsets_match_reference_layout(small_cases):
    cds = small_cases["ragged"]
    wptr, uptr, wsko, usko, total = cds.offsets(3)
    assert np.array_equal(wptr, np.concatenate([[0], np.cumsum(cds.Ddim[:-1])]) * 3)
    assert total == int(cds.slen.sum()) * 3
