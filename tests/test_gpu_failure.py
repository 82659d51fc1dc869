"""GPU: failure detection without a fault.  A host-set test hook makes one CTA withhold a
pipeline stage so a bounded wait of the tensor-core kernel runs out (short limit); the
kernel gives up cleanly, the plan reports MXB_ERR_TIMEOUT, and the same plan then computes
correctly: the context stays usable."""
import numpy as np
import pytest

import oracle as O
from matrox_ru_b200 import _lib, hgemm as H

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as t
    assert t.cuda.is_available(), "GPU tests need a CUDA device"
    from matrox_ru_b200 import build
    build.build()
    return t


def test_wait_that_runs_out_reports_timeout(torch, small_cases):
    cds = small_cases["h2b"]
    r = 64
    TW = np.random.default_rng(0).standard_normal(cds.n * r)
    want = O.eval_h2b(cds, TW, r)
    plan = H.Plan(cds, "split_bf16")
    tw = torch.as_tensor(TW, device="cuda")
    plan.set_test_hooks(_lib.DEBUG_STALL_ONE_WAIT, wait_cycles=100_000_000)  # ~50 ms limit
    plan.evaluate(tw, r)
    with pytest.raises(_lib.MxbError) as e:
        plan.status()
    assert e.value.code == _lib.MXB_ERR_TIMEOUT
    plan.set_test_hooks(0)
    got = plan.evaluate(tw, r).cpu().numpy()
    plan.status()  # cleared, no new error
    assert np.linalg.norm(got - want) / np.linalg.norm(want) <= 1e-5


def test_hooks_rejected_on_fp64_plans(torch, small_cases):
    plan = H.Plan(small_cases["hss"], "fp64")
    with pytest.raises(_lib.MxbError) as e:
        plan.set_test_hooks(_lib.DEBUG_STALL_ONE_WAIT)
    assert e.value.code == _lib.MXB_ERR_UNSUPPORTED


@pytest.mark.parametrize("dataflow", ["1", "0"])
def test_chained_levels_match_separate_launches(torch, small_cases, monkeypatch, dataflow):
    """Up-sweep heights (and down-sweep depths with leaf down) run as one launch each, the
    levels waiting for each other on the device -- node by node through per-node counters
    (dataflow, the default) or level by level (MXB_TC_DATAFLOW=0): the same result as the
    separate launches (the evaluation is exact in the chaining; only the tile schedule
    changes), and fewer launches."""
    import os
    monkeypatch.setenv("MXB_TC_DATAFLOW", dataflow)
    for name in ("h2b", "hss", "ragged"):
        cds = small_cases[name]
        r = 200
        TW = torch.as_tensor(np.random.default_rng(3).standard_normal(cds.n * r), device="cuda")
        # the default tiles, one launch per level
        os.environ["MXB_TC_CHAIN"], os.environ["MXB_AUTOTUNE"] = "0", "0"
        try:
            sep = H.Plan(cds, "split_bf16")
            want = sep.evaluate(TW, r).clone()
            sep.status()
        finally:
            del os.environ["MXB_TC_CHAIN"], os.environ["MXB_AUTOTUNE"]
        n_sep = sep.info()["launches"]
        # the same tiles, levels chained: the same products in the same order, bit-identical
        ch = H.Plan(cds, "split_bf16")
        ch.set_test_hooks(_lib.DEBUG_CHAIN_LEVELS)
        got = ch.evaluate(TW, r)
        ch.status()
        assert ch.info()["launches"] < n_sep, name
        assert torch.equal(got, want), name
        oracle = O.eval_h2b(cds, TW.cpu().numpy(), r)
        err = np.linalg.norm(got.cpu().numpy() - oracle) / np.linalg.norm(oracle)
        assert err <= 1e-5, (name, err)
        prof = ch.profile(TW, r)
        assert any(x["chained"] for x in prof)
        assert all(x["ms"] == 0.0 for x in prof if x["chained"])


@pytest.mark.parametrize("dataflow", ["1", "0"])
def test_level_barrier_that_runs_out_reports_timeout(torch, small_cases, monkeypatch, dataflow):
    """The first level of a chained launch (dataflow: the units without inputs in the launch)
    never reports its units done (test hook): the next level's bounded wait runs out, the plan
    reports MXB_ERR_TIMEOUT, and the same plan then computes correctly."""
    monkeypatch.setenv("MXB_TC_DATAFLOW", dataflow)
    cds = small_cases["h2b"]
    r = 64
    TW = np.random.default_rng(4).standard_normal(cds.n * r)
    want = O.eval_h2b(cds, TW, r)
    plan = H.Plan(cds, "split_bf16")
    tw = torch.as_tensor(TW, device="cuda")
    plan.set_test_hooks(_lib.DEBUG_STALL_LEVEL, wait_cycles=100_000_000)  # ~50 ms limit
    plan.evaluate(tw, r)
    with pytest.raises(_lib.MxbError) as e:
        plan.status()
    assert e.value.code == _lib.MXB_ERR_TIMEOUT
    plan.set_test_hooks(0)
    got = plan.evaluate(tw, r).cpu().numpy()
    plan.status()
    assert np.linalg.norm(got - want) / np.linalg.norm(want) <= 1e-5


def test_one_launch_plan_and_its_level_barrier(torch, small_cases):
    """A plan evaluated as one launch (test hook MXB_DEBUG_ONE_LAUNCH) matches its ordinary
    evaluation; with MXB_DEBUG_STALL_LEVEL added, the first level never reports done, the
    next level's bounded wait runs out, MXB_ERR_TIMEOUT is reported, and the plan recovers."""
    cds = small_cases["h2b"]
    r = 96
    TW = np.random.default_rng(6).standard_normal(cds.n * r)
    want = O.eval_h2b(cds, TW, r)
    tw = torch.as_tensor(TW, device="cuda")
    plan = H.Plan(cds, "split_bf16")
    plan.set_test_hooks(_lib.DEBUG_ONE_LAUNCH)
    got = plan.evaluate(tw, r).cpu().numpy()
    plan.status()
    assert plan.info()["launches"] == 1
    assert np.linalg.norm(got - want) / np.linalg.norm(want) <= 1e-5
    plan.set_test_hooks(_lib.DEBUG_ONE_LAUNCH | _lib.DEBUG_STALL_LEVEL, wait_cycles=100_000_000)
    plan.evaluate(tw, r)
    with pytest.raises(_lib.MxbError) as e:
        plan.status()
    assert e.value.code == _lib.MXB_ERR_TIMEOUT
    plan.set_test_hooks(0)
    again = plan.evaluate(tw, r).cpu().numpy()
    plan.status()
    assert np.linalg.norm(again - want) / np.linalg.norm(want) <= 1e-5
