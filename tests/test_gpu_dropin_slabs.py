"""GPU: the reference-signature drop-ins evaluate in column slabs whose host<->device copies
overlap the evaluation of neighbouring slabs.  These cases reach several slabs (more than the
two slab buffers in rotation), a narrower last slab, leaf blocks that the caller spaces
unevenly in its arrays, and every output semantics (H2-b accumulate, H2-b into a zero output,
HSS overwrite), against the oracle."""
import numpy as np
import pytest

import oracle as O
from conftest import rel_err
from matrox_ru_b200 import _lib, hgemm as H

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as t
    assert t.cuda.is_available(), "GPU tests need a CUDA device"
    from matrox_ru_b200 import build
    build.build()
    return t


@pytest.fixture(autouse=True)
def _defaults(torch):
    H.set_precision("fp64")
    H.set_flags(0)
    yield
    H.set_precision("fp64")
    H.set_flags(0)


class Spaced:
    """A CDS whose leaf blocks sit `gap` elements apart in the caller's W / Y arrays, the
    first block at offset `lead` (the reference's wptr / uptr are free offsets)."""

    def __init__(self, cds, lead, gap):
        self.__dict__.update(_cds=cds, lead=lead, gap=gap)

    def __getattr__(self, k):
        return getattr(self._cds, k)

    def offsets(self, nrhs):
        wptr, uptr, wsko, usko, rest = self._cds.offsets(nrhs)
        add = self.lead + np.arange(len(wptr), dtype=np.int64) * self.gap
        return (wptr + add).astype(np.int32), (uptr + add).astype(np.int32), wsko, usko, rest

    def spread(self, packed, nrhs, fill):
        wptr, _, _, _, _ = self.offsets(nrhs)
        out = np.full(int(wptr[-1]) + int(self.Ddim[-1]) * nrhs + self.gap, fill)
        for i in range(self.nleaf):
            a, b = int(self.leaf_lids_offset[i]), int(self.leaf_lids_offset[i + 1])
            out[wptr[i]:wptr[i] + (b - a) * nrhs] = packed[a * nrhs:b * nrhs]
        return out

    def gather(self, spread, nrhs):
        wptr, _, _, _, _ = self.offsets(nrhs)
        out = np.empty(self.n * nrhs)
        for i in range(self.nleaf):
            a, b = int(self.leaf_lids_offset[i]), int(self.leaf_lids_offset[i + 1])
            out[a * nrhs:b * nrhs] = spread[wptr[i]:wptr[i] + (b - a) * nrhs]
        return out


@pytest.mark.parametrize("nrhs", [1030, 300])
@pytest.mark.parametrize("name", ["h2b", "ragged"])
def test_h2b_slabs_accumulate(torch, small_cases, name, nrhs):
    cds = small_cases[name]
    rng = np.random.default_rng(nrhs)
    TW = rng.standard_normal(cds.n * nrhs)
    Y0 = rng.standard_normal(cds.n * nrhs)
    want = Y0 + O.eval_h2b(cds, TW, nrhs)
    got = Y0.copy()
    H.CBHGEMM(cds, TW, got, nrhs)
    assert rel_err(got, want) <= 1e-12


@pytest.mark.parametrize("name", ["h2b", "ragged"])
def test_h2b_slabs_spaced_blocks(torch, small_cases, name):
    """Unevenly spaced leaf blocks: runs of equal leaves move as 2-D copies, the rest one by
    one; nothing outside the blocks is written."""
    cds = small_cases[name]
    nrhs = 515
    for lead, gap in ((0, 37), (5, 0)):
        sp = Spaced(cds, lead, gap)
        rng = np.random.default_rng(gap)
        TW = rng.standard_normal(cds.n * nrhs)
        Y0 = rng.standard_normal(cds.n * nrhs)
        want = Y0 + O.eval_h2b(cds, TW, nrhs)
        TWs = sp.spread(TW, nrhs, np.nan)
        Ys = sp.spread(Y0, nrhs, -7.0)
        H.CBHGEMM(sp, TWs, Ys, nrhs)
        assert rel_err(sp.gather(Ys, nrhs), want) <= 1e-12
        mask = np.isnan(TWs)
        assert np.all(Ys[mask] == -7.0)


def test_h2b_slabs_zero_output_flag(torch, small_cases):
    cds = small_cases["h2b"]
    nrhs = 777
    TW = np.random.default_rng(3).standard_normal(cds.n * nrhs)
    want = O.eval_h2b(cds, TW, nrhs)
    got = np.full_like(TW, np.nan)  # not read: the caller declared it zero
    H.set_flags(_lib.FLAG_OUTPUT_IS_ZERO)
    H.CBHGEMM(cds, TW, got, nrhs)
    assert rel_err(got, want) <= 1e-12


def test_hss_slabs_overwrite(torch, small_cases):
    cds = small_cases["hss"]
    nrhs = 1100
    TW = np.random.default_rng(4).standard_normal(cds.n * nrhs)
    want = O.eval_h2b(cds, TW, nrhs)  # HSS CDS: overwrite semantics
    got = np.full_like(TW, 3.0)
    H.parHSSGEMM(cds, TW, got, nrhs)
    assert rel_err(got, want) <= 1e-12


@pytest.mark.parametrize("mode", ["split_bf16", "split_bf16_x6"])
def test_split_slabs_match_plan(torch, small_cases, mode):
    """Split-BF16 drop-in in slabs vs the same plan on all columns at once."""
    cds = small_cases["h2b"]
    nrhs = 640
    TW = np.random.default_rng(5).standard_normal(cds.n * nrhs)
    want = O.eval_h2b(cds, TW, nrhs)
    H.set_precision(mode)
    got = np.zeros_like(TW)
    H.CBHGEMM(cds, TW, got, nrhs)
    whole = H.Plan(cds, mode).evaluate(torch.as_tensor(TW, device="cuda"), nrhs).cpu().numpy()
    err = np.linalg.norm(got - want) / np.linalg.norm(want)
    assert 1e-12 < err <= 1e-5
    assert np.linalg.norm(got - whole) / np.linalg.norm(whole) <= 1e-5
