"""CPU: the reference's own host pipeline as the source of truth for the structure format,
the structure builder and the oracle.

The fixtures ``tests/golden/ref_pipeline/*.npz`` (``tests/golden/make_ref_pipeline.py``) hold
what the REFERENCE's code produced for seeded points: the structure generator's ``.bin`` files
(``sympiler/HTree.cpp:469-543``), the CDS exactly as ``DUV2CDS`` packs it
(``matroxTest-V1/hcds.h:433-460``), and the outputs of the evaluator the generator emitted for
that structure and of ``CBHGEMM`` / ``parHSSGEMM``.
"""
import glob
import os

import numpy as np
import pytest

import oracle as O
import ref_pipeline as RP
from matrox_ru_b200 import structure as S, structure_bin as SB

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURES = sorted(glob.glob(os.path.join(HERE, "golden", "ref_pipeline", "*.npz")))


def load(path):
    z = np.load(path)
    arrays = {k[4:]: z[k] for k in z.files if k.startswith("cds/")}
    scalars = {k: int(v) for k, v in z["scalars"]}
    files = {k[7:]: z[k] for k in z.files if k.startswith("struct/")}
    return z, RP.cds_from_dump(arrays, scalars), arrays, files


def write_files(files, directory):
    for name, a in files.items():
        a.tofile(os.path.join(directory, name))


def test_fixture_set_covers_hss_and_h2b():
    kinds = {bool(load(p)[1].is_hss) for p in FIXTURES}
    assert kinds == {True, False}


@pytest.mark.parametrize("path", FIXTURES, ids=os.path.basename)
def test_reader_reads_the_generators_files(path, tmp_path):
    """read_structure on the files the reference's generator wrote, and structure_arrays back:
    every file is reproduced exactly (tree, level sets, coarsening, blocking, k-NN lists)."""
    z, cds, arrays, files = load(path)
    write_files(files, str(tmp_path))
    st = SB.read_structure(str(tmp_path), z["X"])
    assert st.is_hss == cds.is_hss
    assert st.NN is not None and st.NN.size == 32 * cds.n
    back = SB.structure_arrays(st)
    for name, a in files.items():
        assert name in back, name
        assert np.array_equal(np.asarray(back[name]).astype(a.dtype), a), name


@pytest.mark.parametrize("path", FIXTURES, ids=os.path.basename)
def test_builder_matches_the_generators_tree_and_lists(path, tmp_path):
    """structure.py's own tree and interaction lists equal the generator's: the same point
    set in every node, the same near and far lists, the same coarsening and blocking."""
    z, cds, arrays, files = load(path)
    budget, leaf = float(z["params"][0]), int(z["params"][1])
    write_files(files, str(tmp_path))
    ref = SB.read_structure(str(tmp_path), z["X"])
    ours = SB.build_structure(z["X"], leaf, budget)
    for v in range(1, ref.tree.numnodes):
        assert np.array_equal(np.sort(ref.tree.lids[v]), np.sort(ours.tree.lids[v])), v
    assert ref.near == ours.near
    assert ref.far == ours.far
    mine = SB.structure_arrays(ours)
    for name in ("dim.bin", "levelset.bin", "idx.bin", "cidx.bin", "wpart.bin", "clevelset.bin", "nxval.bin",
                 "nyval.bin", "fxval.bin", "fyval.bin", "nblockset.bin", "nblocks.bin", "fblockset.bin",
                 "fblocks.bin", "leafmap.bin", "lchildren.bin", "rchildren.bin", "lidsoffset.bin", "lidslen.bin"):
        if name in files:
            assert np.array_equal(np.asarray(mine[name]).astype(np.int32), files[name]), name


@pytest.mark.parametrize("path", FIXTURES, ids=os.path.basename)
def test_reference_cds_layout(path):
    """The reference's CDS is what the drop-in receives: check the arrays it relies on."""
    z, cds, arrays, files = load(path)
    nn = cds.numnodes
    assert np.array_equal(cds.cidx, files["cidx.bin"])
    assert np.array_equal(np.sort(cds.cidx), np.arange(1, nn))
    # block rows as the reference's readHtree counts them: one fewer than the offset arrays
    if not cds.is_hss:
        assert cds.nrow == len(files["nblockset.bin"]) - 1
        assert cds.frow == len(files["fblockset.bin"]) - 1
    # every block lies inside its pool
    ends = cds.Dptr.astype(np.int64) + cds.Ddim[cds.npairx].astype(np.int64) * cds.Ddim[cds.npairy]
    assert ends.max() == cds.D.size
    if cds.fcount:
        ends = cds.Bptr.astype(np.int64) + cds.slen[cds.fpairx].astype(np.int64) * cds.slen[cds.fpairy]
        assert ends.max() == cds.B.size


@pytest.mark.parametrize("path", FIXTURES, ids=os.path.basename)
def test_oracle_on_the_reference_cds(path):
    """The oracle's restatement reproduces the generated evaluator and the structure-generic
    reference evaluator on the reference's own CDS."""
    z, cds, arrays, files = load(path)
    r = int(z["nrhs"][0])
    Yg, Ys = z["Y_generated"], z["Y_structure_generic"]
    assert np.abs(Yg - Ys).max() <= 1e-12 * np.abs(Ys).max()
    got = O.eval_h2b(cds, z["TW"], r)
    assert np.abs(got - Yg).max() <= 1e-13 * np.abs(Yg).max()
    if O.ref_available():
        live = O.eval_h2b(cds, z["TW"], r, use_reference=True)
        assert np.abs(live - Ys).max() <= 1e-13 * np.abs(Ys).max()


@pytest.mark.skipif(not RP.available(), reason="reference pipeline binaries not built")
@pytest.mark.parametrize("path", FIXTURES, ids=os.path.basename)
def test_reference_pipeline_reproduces_the_fixture(path, tmp_path):
    """Run live, the reference pipeline (one thread) makes the fixture's CDS again."""
    z, cds, arrays, files = load(path)
    budget, leaf, tol, h, mr = z["params"]
    run = RP.run(z["X"], budget=budget, leaf=int(leaf), tol=tol, h=h, max_rank=int(mr), threads=1,
                 workdir=str(tmp_path))
    for name, a in arrays.items():
        assert np.array_equal(run.arrays[name], a), name


@pytest.mark.parametrize("path", FIXTURES, ids=os.path.basename)
def test_producer_reproduces_the_reference_compression(path, tmp_path):
    """structure.build_cds on the generator's files (its tree, lists and 32-NN lists), with
    the reference's k-NN sampling and the reference's rand() sequence (one thread), makes the
    reference's CDS: the same ranks, the same skeleton points in the same order, the same
    blocks up to kernel rounding, and the same evaluation."""
    from glibc_rand import GlibcRand
    z, ref, arrays, files = load(path)
    budget, leaf, tol, h, mr = z["params"]
    write_files(files, str(tmp_path))
    st = SB.read_structure(str(tmp_path), z["X"])
    ours = S.build_cds(z["X"], S.KernelSpec("gaussian", h), leaf_size=int(leaf), budget=budget, tol=tol,
                       max_rank=int(mr), structure=st, rand_source=GlibcRand())
    assert np.array_equal(ours.slen, ref.slen)
    for v in range(1, ref.numnodes):
        assert np.array_equal(ours.skels[v], ref.skels[v]), v
    for name in ("npairx", "npairy", "fpairx", "fpairy", "nblockset", "nblocks", "fblockset", "fblocks",
                 "Ddim", "lchildren", "rchildren", "levelset", "idx", "cidx", "wpart", "clevelset"):
        assert np.array_equal(getattr(ours, name), getattr(ref, name)), name
    # blocks: the layouts of the pools may differ, compare block by block
    for k in range(ref.ncount):
        m = int(ref.Ddim[ref.npairx[k]]) * int(ref.Ddim[ref.npairy[k]])
        a = ours.D[int(ours.Dptr[k]):int(ours.Dptr[k]) + m]
        b = ref.D[int(ref.Dptr[k]):int(ref.Dptr[k]) + m]
        assert np.abs(a - b).max() <= 1e-13
    for k in range(ref.fcount):
        m = int(ref.slen[ref.fpairx[k]]) * int(ref.slen[ref.fpairy[k]])
        a = ours.B[int(ours.Bptr[k]):int(ours.Bptr[k]) + m]
        b = ref.B[int(ref.Bptr[k]):int(ref.Bptr[k]) + m]
        assert np.abs(a - b).max() <= 1e-13
    scale = np.abs(ref.VT).max()
    for v in range(1, ref.numnodes):
        m = int(ref.slen[v]) * int(arrays["proj_column"][v])
        a = ours.VT[int(ours.VTptr[v]):int(ours.VTptr[v]) + m]
        b = ref.VT[int(ref.VTptr[v]):int(ref.VTptr[v]) + m]
        assert np.abs(a - b).max() <= 1e-10 * scale, v
    r = int(z["nrhs"][0])
    got = O.eval_h2b(ours, z["TW"], r)
    assert np.abs(got - z["Y_generated"]).max() <= 1e-11 * np.abs(z["Y_generated"]).max()


def test_glibc_rand_restatement_matches_libc():
    """The oracle's restatement of rand() (default seed) against the C library here."""
    import ctypes
    from glibc_rand import GlibcRand
    libc = ctypes.CDLL("libc.so.6")
    libc.srand(1)
    g = GlibcRand()
    assert all(g() == libc.rand() for _ in range(20000))
