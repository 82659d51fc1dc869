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
