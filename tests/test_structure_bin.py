"""CPU: the reference's on-disk structure format (sympiler/HTree.cpp:468-542 writes it,
matroxTest-V1/HTree.h:76-243 reads it).  Files, dtypes and lengths follow the writer; a
structure written here reads back identically, and the CDS compressed on the read structure
is identical to the CDS built directly, array for array."""
import os

import numpy as np
import pytest

import oracle as O
from matrox_ru_b200 import structure as S, structure_bin as B


def case(name):
    if name == "h2b":
        X = S.gaussian_mixture(768, 4, 4, 0.0, 3.0, 0.4, None, seed=12)
        return X, dict(leaf_size=48, budget=0.25), dict(tol=1e-6, max_rank=40)
    if name == "hss":
        X = S.gaussian_mixture(512, 3, 4, 0.0, 3.0, 0.4, None, seed=11)
        return X, dict(leaf_size=32, budget=0.0), dict(tol=1e-6, max_rank=24)
    X = S.gaussian_mixture(700, 5, 6, -1.0, 1.0, 0.3, 0.8, seed=13)  # ragged leaves
    return X, dict(leaf_size=40, budget=0.2), dict(tol=1e-5, max_rank=32)


@pytest.mark.parametrize("name", ["h2b", "hss", "ragged"])
def test_files_follow_the_reference_writer(tmp_path, name):
    X, sargs, _ = case(name)
    st = B.build_structure(X, **sargs)
    names = B.write_structure(st, str(tmp_path))
    t = st.tree
    size = lambda f: os.path.getsize(tmp_path / f) // (8 if f == "distNN.bin" else 4)
    assert set(names) <= set(B.FILES)
    assert set(B.BLOCK_FILES) <= set(names) or st.is_hss
    assert size("dim.bin") == t.nleaf
    for f in ("leafmap.bin", "lidsoffset.bin", "lidslen.bin", "lchildren.bin", "rchildren.bin"):
        assert size(f) == t.numnodes, f
    assert size("levelset.bin") == t.depth + 1
    assert size("idx.bin") == size("cidx.bin") == t.numnodes - 1
    assert size("lids.bin") == sum(len(t.lids[v]) for v in range(1, t.numnodes))
    lm = np.fromfile(tmp_path / "leafmap.bin", dtype="<i4")
    assert (lm[:t.first_leaf] == -1).all() and (lm[t.first_leaf:] == np.arange(t.nleaf)).all()


@pytest.mark.parametrize("name", ["h2b", "hss", "ragged"])
def test_round_trip_and_cds(tmp_path, name):
    X, sargs, cargs = case(name)
    st = B.build_structure(X, **sargs)
    B.write_structure(st, str(tmp_path))
    rd = B.read_structure(str(tmp_path), X)
    assert rd.near == st.near and rd.far == st.far
    for v in range(1, st.tree.numnodes):
        assert np.array_equal(rd.tree.lids[v], st.tree.lids[v])
    assert np.array_equal(rd.tree.mid, st.tree.mid) and np.array_equal(rd.tree.radius, st.tree.radius)
    a, b = B.structure_arrays(st), B.structure_arrays(rd)
    assert a.keys() == b.keys() and all(np.array_equal(a[k], b[k]) for k in a)
    direct = S.build_cds(X, S.KernelSpec("gaussian", 1.0), leaf_size=sargs["leaf_size"], budget=sargs["budget"], **cargs)
    imported = S.build_cds(X, S.KernelSpec("gaussian", 1.0), leaf_size=sargs["leaf_size"], structure=rd, **cargs)
    for k in S.CDS._ARRAYS:
        assert np.array_equal(getattr(direct, k), getattr(imported, k)), k
    r = 3
    W = np.random.default_rng(0).standard_normal(direct.n * r)
    assert np.array_equal(O.eval_h2b(direct, W, r), O.eval_h2b(imported, W, r))


def test_reader_rejects_bad_structures(tmp_path):
    X, sargs, _ = case("h2b")
    st = B.build_structure(X, **sargs)
    B.write_structure(st, str(tmp_path))
    lch = np.fromfile(tmp_path / "lchildren.bin", dtype="<i4")
    lch[0] = 5
    lch.tofile(tmp_path / "lchildren.bin")
    with pytest.raises(ValueError, match="heap numbering"):
        B.read_structure(str(tmp_path), X)
    B.write_structure(st, str(tmp_path))
    lids = np.fromfile(tmp_path / "lids.bin", dtype="<i4")
    lids[0] = X.shape[0] + 3
    lids.tofile(tmp_path / "lids.bin")
    with pytest.raises(ValueError, match="point id"):
        B.read_structure(str(tmp_path), X)
    B.write_structure(st, str(tmp_path))
    os.remove(tmp_path / "dim.bin")
    with pytest.raises(FileNotFoundError):
        B.read_structure(str(tmp_path), X)


def test_nn_lists_round_trip(tmp_path):
    """NN.bin (int32) and distNN.bin (float64, one distance per NN entry) as the reference's
    reader expects them (matroxTest-V1/HTree.h:78-94)."""
    X, sargs, _ = case("hss")
    st = B.build_structure(X, **sargs)
    k = 4
    d2 = S.sqdist(X, X)
    np.fill_diagonal(d2, np.inf)
    nn = np.argsort(d2, axis=1, kind="stable")[:, :k]
    st.NN = nn.reshape(-1)
    st.distNN = np.sqrt(np.take_along_axis(d2, nn, axis=1)).reshape(-1)
    B.write_structure(st, str(tmp_path))
    assert os.path.getsize(tmp_path / "distNN.bin") == 2 * os.path.getsize(tmp_path / "NN.bin")
    rd = B.read_structure(str(tmp_path), X)
    assert np.array_equal(rd.NN, st.NN) and np.array_equal(rd.distNN, st.distNN)
