"""GPU: launch-by-launch timing (mxb_plan_profile / mxb_batch_profile).  The per-launch
algorithmic flops must add up exactly to the reference's flop model (computeFlops,
matroxTest-V1/compression.h:1079-1130, restated by mxb_plan_flops), and the profiled
evaluation must leave the ordinary result in Y."""
import numpy as np
import pytest

from matrox_ru_b200 import hgemm as H

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as t
    assert t.cuda.is_available(), "GPU tests need a CUDA device"
    from matrox_ru_b200 import build
    build.build()
    return t


@pytest.mark.parametrize("precision", ["fp64", "split_bf16", "split_bf16_far6", "split_bf16_x6"])
@pytest.mark.parametrize("name", ["hss", "h2b", "ragged"])
def test_profile_flops_and_result(torch, small_cases, name, precision):
    cds = small_cases[name]
    r = 72
    plan = H.Plan(cds, precision)
    g = torch.Generator(device="cuda")
    g.manual_seed(5)
    TW = torch.randn(cds.n * r, dtype=torch.float64, device="cuda", generator=g)
    want = plan.evaluate(TW, r)
    out = torch.full_like(want, 7.0)  # overwritten by the profiled evaluation
    recs = plan.profile(TW, r, out=out)
    torch.cuda.synchronize()
    plan.status()
    # one record per op; ops chained into the launch before them (device-side level barriers)
    # report ms 0, the launch's own record covers them
    assert sum(not x["chained"] for x in recs) == plan.info()["launches"]
    assert sum(x["flops"] for x in recs) == plan.flops(r) == cds.flops(r)
    for x in recs:
        assert (x["ms"] > 0.0) != x["chained"]
        assert x["issued_flops"] >= x["flops"]
        assert x["units"] > 0 or x["flops"] == 0  # units without items zero their output
    phases = {x["phase"] for x in recs}
    if precision == "fp64":
        assert phases <= {"up", "far_down", "near_leaf_down"}
    else:
        assert phases <= {"split_w", "up", "far", "far_near", "down", "near", "leaf_down"}
        # the far couplings of all depths run as one launch, joined by the near field when
        # both use the same number of products
        assert sum(x["phase"] in ("far", "far_near") for x in recs) == 1
        assert ("near" in phases) == (precision == "split_bf16_far6")
        k = 6.0 if precision == "split_bf16_x6" else None
        if k:
            for x in recs:
                assert x["issued_flops"] >= k * x["flops"]
    torch.testing.assert_close(out, want, rtol=1e-13, atol=1e-13 * float(want.abs().max()))


def test_batch_profile(torch, small_cases):
    cases = [(small_cases["h2b"], 40), (small_cases["ragged"], 200), (small_cases["hss"], 96)]
    plans = [H.Plan(c, "split_bf16") for c, _ in cases]
    batch = H.Batch(plans)
    TWs = [torch.randn(c.n * r, dtype=torch.float64, device="cuda") for c, r in cases]
    want = batch.evaluate(TWs, [r for _, r in cases])
    outs = [torch.zeros_like(w) for w in want]
    recs = batch.profile(TWs, [r for _, r in cases], outs)
    batch.status()
    assert sum(not x["chained"] for x in recs) == batch.info()["launches"]
    assert sum(x["flops"] for x in recs) == sum(c.flops(r) for c, r in cases)
    for o, w in zip(outs, want):
        torch.testing.assert_close(o, w, rtol=1e-13, atol=1e-13 * float(w.abs().max()))
