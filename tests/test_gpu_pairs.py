"""GPU: the split-BF16 tensor-core kernel on pairs of SMs (2-CTA clusters, 256-row tiles,
tcgen05.mma.cta_group::2), forced on every launch with MXB_TC_TILE, against the FP64 oracle.

The cases have output blocks taller than 128 rows (leaves of up to 256 points, ranks up to
~180), so both CTAs of a pair hold real rows, plus blocks of at most 128 rows where the odd
CTA's rows are all padding.  The failure hook checks that a wait that runs out in a pair ends
both CTAs cleanly."""
import os

import numpy as np
import pytest

import oracle as O
from matrox_ru_b200 import _lib, hgemm as H, structure as S

pytestmark = pytest.mark.gpu
PAIR = _lib.TILE_PAIR


@pytest.fixture(scope="module")
def torch():
    import torch as t
    assert t.cuda.is_available(), "GPU tests need a CUDA device"
    from matrox_ru_b200 import build
    build.build()
    return t


@pytest.fixture(scope="module")
def tall_cases():
    out = {}
    X = S.gaussian_mixture(3000, 6, 5, -1.0, 1.0, 0.3, 0.8, seed=21)
    out["h2b_tall"] = S.build_cds(X, S.KernelSpec("gaussian", 1.2), leaf_size=256, budget=0.2, tol=1e-9,
                                  max_rank=180, seed=1)
    X = S.gaussian_mixture(2048, 4, 4, 0.0, 3.0, 0.4, None, seed=22)
    out["hss_tall"] = S.build_cds(X, S.KernelSpec("imq", 1.0), leaf_size=256, budget=0.0, tol=1e-9,
                                  max_rank=200, seed=2)
    return out


@pytest.fixture
def forced_tile():
    old = os.environ.get("MXB_TC_TILE")

    def set_tile(code):
        os.environ["MXB_TC_TILE"] = str(code)

    yield set_tile
    if old is None:
        os.environ.pop("MXB_TC_TILE", None)
    else:
        os.environ["MXB_TC_TILE"] = old


def frob(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_cases_have_tall_blocks(tall_cases):
    for cds in tall_cases.values():
        assert max(cds.Ddim) > 128 and max(cds.slen) > 128


@pytest.mark.parametrize("mode", ["split_bf16", "split_bf16_x6"])
@pytest.mark.parametrize("tile", [256 | PAIR, 128 | PAIR])
@pytest.mark.parametrize("name", ["h2b_tall", "hss_tall"])
def test_pairs_match_fp64(torch, tall_cases, forced_tile, name, tile, mode):
    cds = tall_cases[name]
    forced_tile(tile)
    plan = H.Plan(cds, mode)
    for r, seed in ((300, 3), (40, 4)):
        TW = np.random.default_rng(seed).standard_normal(cds.n * r)
        want = O.eval_h2b(cds, TW, r)
        tw = torch.as_tensor(TW, device="cuda")
        got = plan.evaluate(tw, r)
        plan.status()
        err = frob(got.cpu().numpy(), want)
        assert 1e-12 < err <= (1e-5 if mode == "split_bf16" else 5e-6), (r, err)
        recs = plan.profile(tw, r)
        plan.status()
        assert all(x["pair"] for x in recs if x["phase"] != "split_w")
        assert sum(x["flops"] for x in recs) == cds.flops(r)


def test_pairs_agree_with_single_ctas(torch, tall_cases, forced_tile):
    cds = tall_cases["h2b_tall"]
    r = 256
    tw = torch.as_tensor(np.random.default_rng(7).standard_normal(cds.n * r), device="cuda")
    forced_tile(128)
    single = H.Plan(cds, "split_bf16").evaluate(tw, r).cpu().numpy()
    forced_tile(256 | PAIR)
    pair = H.Plan(cds, "split_bf16").evaluate(tw, r).cpu().numpy()
    assert frob(pair, single) <= 2e-6


def test_pair_wait_that_runs_out_reports_timeout(torch, tall_cases, forced_tile):
    cds = tall_cases["h2b_tall"]
    r = 64
    TW = np.random.default_rng(0).standard_normal(cds.n * r)
    want = O.eval_h2b(cds, TW, r)
    forced_tile(256 | PAIR)
    plan = H.Plan(cds, "split_bf16")
    tw = torch.as_tensor(TW, device="cuda")
    plan.set_test_hooks(_lib.DEBUG_STALL_ONE_WAIT, wait_cycles=100_000_000)  # ~50 ms limit
    plan.evaluate(tw, r)
    with pytest.raises(_lib.MxbError) as e:
        plan.status()
    assert e.value.code == _lib.MXB_ERR_TIMEOUT
    plan.set_test_hooks(0)
    got = plan.evaluate(tw, r).cpu().numpy()
    plan.status()
    assert frob(got, want) <= 1e-5


@pytest.mark.parametrize("name", ["ragged", "hss"])
def test_pairs_on_short_blocks(torch, small_cases, forced_tile, name):
    """Blocks of at most 128 rows: the odd CTA of every pair stages no A and stores nothing."""
    cds = small_cases[name]
    forced_tile(256 | PAIR)
    r = 130
    TW = np.random.default_rng(5).standard_normal(cds.n * r)
    want = O.eval_h2b(cds, TW, r)
    plan = H.Plan(cds, "split_bf16")
    got = plan.evaluate(torch.as_tensor(TW, device="cuda"), r)
    plan.status()
    assert 1e-12 < frob(got.cpu().numpy(), want) <= 1e-5
