"""GPU: batches of uneven H-matrices (the 64-matrix batch workload, scaled down): different N, point
dimension, kernel (Gaussian / inverse multiquadric), ranks and nrhs, evaluated by one merged
launch sequence with autotuned column tiles; each result is checked against the FP64 oracle."""
import numpy as np
import pytest

import oracle as O
from matrox_ru_b200 import hgemm as H, structure as S

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as t
    assert t.cuda.is_available(), "GPU tests need a CUDA device"
    from matrox_ru_b200 import build
    build.build()
    return t


def make_cases(count, seed):
    rng = np.random.default_rng(seed)
    cases = []
    for i in range(count):
        n = int(np.exp(rng.uniform(np.log(600), np.log(4000))))
        d = int(rng.choice([3, 5, 8]))
        kind = "gaussian" if i % 2 == 0 else "imq"
        h = float(rng.uniform(0.7, 2.0))
        X = S.gaussian_mixture(n, d, 4, -1.0, 1.0, 0.3, 0.8, seed=seed * 100 + i)
        cds = S.build_cds(X, S.KernelSpec(kind, h), leaf_size=int(rng.choice([64, 128])),
                          budget=float(rng.choice([0.0, 0.2])), tol=1e-5, max_rank=48, seed=i)
        r = int(np.exp(rng.uniform(np.log(16), np.log(300))))
        cases.append((cds, r))
    return cases


def test_batch_matches_oracle_and_single_plans(torch):
    cases = make_cases(6, seed=3)
    plans = [H.Plan(c, "split_bf16") for c, _ in cases]
    batch = H.Batch(plans)
    TWs, wants = [], []
    for k, (c, r) in enumerate(cases):
        TW = np.random.default_rng(k).standard_normal(c.n * r)
        TWs.append(torch.as_tensor(TW, device="cuda"))
        wants.append(O.eval_h2b(c, TW, r))
    nrhs = [r for _, r in cases]
    for rep in range(2):  # the second evaluation replays the captured graph
        outs = batch.evaluate(TWs, nrhs)
        batch.status()
        for (c, r), o, want in zip(cases, outs, wants):
            err = np.linalg.norm(o.cpu().numpy() - want) / np.linalg.norm(want)
            assert 1e-12 < err <= 1e-5, (rep, c.n, r, err)
    info = batch.info()
    assert info["widths"] and set(info["widths"]) <= {64, 128, 256}
    # a single plan evaluated alone agrees with its batched result
    single = plans[0].evaluate(TWs[0], nrhs[0])
    assert np.linalg.norm(single.cpu().numpy() - outs[0].cpu().numpy()) <= 1e-6 * np.linalg.norm(wants[0])


def pick_modes(torch, cases, TWs, kws, margin=8e-6):
    """Per-plan precision, as the batch workload chooses it: the cheapest split mode whose
    error against the FP64 oracle on the plan's own right-hand sides is within the margin."""
    plans, modes = [], []
    for (c, r), tw, kw in zip(cases, TWs, kws):
        for mode in ("split_bf16", "split_bf16_far6", "split_bf16_x6"):
            p = H.Plan(c, mode)
            y = p.evaluate(tw, r).cpu().numpy()
            p.status()
            if np.linalg.norm(y - kw) / np.linalg.norm(kw) <= margin or mode == "split_bf16_x6":
                break
        plans.append(p)
        modes.append(mode)
    return plans, modes


def test_batch_accumulates(torch):
    cases = make_cases(3, seed=5)
    TWs, Y0s, kws = [], [], []
    for k, (c, r) in enumerate(cases):
        TW = np.random.default_rng(10 + k).standard_normal(c.n * r)
        Y0 = np.random.default_rng(20 + k).standard_normal(c.n * r)
        TWs.append(torch.as_tensor(TW, device="cuda"))
        Y0s.append(torch.as_tensor(Y0, device="cuda"))
        kws.append(O.eval_h2b(c, TW, r))
    plans, modes = pick_modes(torch, cases, TWs, kws)
    batch = H.Batch(plans)
    outs = [y.clone() for y in Y0s]
    batch.evaluate(TWs, [r for _, r in cases], outs=outs, accumulate=True)
    batch.status()
    for o, y0, kw, m in zip(outs, Y0s, kws, modes):
        # accumulate = 1 adds, for HSS plans too
        got = o.cpu().numpy() - y0.cpu().numpy()
        assert np.linalg.norm(got - kw) / np.linalg.norm(kw) <= 1e-5, m


def uneven_batch_cases(count, seed):
    """The batch workload's recipe with N scaled down: N log-uniform, d from {8, 18, 28, 54},
    Gaussian (h in [0.5, 3]) or inverse multiquadric kernels, nrhs log-uniform in [32, 512]."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(np.exp(rng.uniform(np.log(512), np.log(2048))))
        d = int(rng.choice([8, 18, 28, 54]))
        kind = "gaussian" if rng.uniform() < 0.5 else "imq"
        h = float(rng.uniform(0.5, 3.0))
        X = S.gaussian_mixture(n, d, 8, -2.0, 2.0, 0.3, 1.0, seed=seed * 1000 + i)
        cds = S.build_cds(X, S.KernelSpec(kind, h), leaf_size=128, budget=0.25, tol=1e-5, max_rank=64, seed=i)
        r = int(np.exp(rng.uniform(np.log(32), np.log(512))))
        out.append((cds, r))
    return out


def test_sixty_four_uneven_matrices_one_sequence(torch):
    cases = uneven_batch_cases(64, seed=9)
    plans = [H.Plan(c, "split_bf16") for c, _ in cases]
    batch = H.Batch(plans)
    per_plan = max(p.info()["launches"] for p in plans)
    assert batch.info()["launches"] <= per_plan + 2  # merged by level, not 64 sequences
    TWs, wants = [], []
    for k, (c, r) in enumerate(cases):
        TW = np.random.default_rng(k).standard_normal(c.n * r)
        TWs.append(torch.as_tensor(TW, device="cuda"))
        wants.append(O.eval_h2b(c, TW, r))
    outs = batch.evaluate(TWs, [r for _, r in cases])
    batch.status()
    errs = [np.linalg.norm(o.cpu().numpy() - w) / np.linalg.norm(w) for o, w in zip(outs, wants)]
    assert max(errs) <= 1e-5, max(errs)


def test_batch_mixes_split_modes(torch):
    """Plans of different split modes share a batch (per-plan precision): couplings with 3
    and 6 products run in separate launches; every result matches its plan evaluated alone."""
    cases = make_cases(5, seed=7)
    modes = ["split_bf16", "split_bf16_far6", "split_bf16", "split_bf16_x6", "split_bf16_far6"]
    plans = [H.Plan(c, m) for (c, _), m in zip(cases, modes)]
    batch = H.Batch(plans)
    TWs, wants = [], []
    for k, (c, r) in enumerate(cases):
        TW = np.random.default_rng(30 + k).standard_normal(c.n * r)
        TWs.append(torch.as_tensor(TW, device="cuda"))
        wants.append(O.eval_h2b(c, TW, r))
    nrhs = [r for _, r in cases]
    outs = batch.evaluate(TWs, nrhs)
    batch.status()
    for (c, r), m, p, tw, o, want in zip(cases, modes, plans, TWs, outs, wants):
        err = np.linalg.norm(o.cpu().numpy() - want) / np.linalg.norm(want)
        assert 1e-12 < err <= (5e-6 if m != "split_bf16" else 1e-5), (m, err)
        alone = p.evaluate(tw, r).cpu().numpy()
        assert np.linalg.norm(alone - o.cpu().numpy()) <= 1e-6 * np.linalg.norm(want), m


def test_one_launch_batch(torch):
    """MXB_BATCH_ONE_LAUNCH: the W split and every level of every plan (mixed split modes
    included) run as ONE launch with device-side level barriers; the results match the oracle
    and the level-launch evaluation of the same batch."""
    cases = make_cases(5, seed=11)
    modes = ["split_bf16", "split_bf16_far6", "split_bf16", "split_bf16_x6", "split_bf16"]
    plans = [H.Plan(c, m) for (c, _), m in zip(cases, modes)]
    TWs, wants = [], []
    for k, (c, r) in enumerate(cases):
        TW = np.random.default_rng(40 + k).standard_normal(c.n * r)
        TWs.append(torch.as_tensor(TW, device="cuda"))
        wants.append(O.eval_h2b(c, TW, r))
    nrhs = [r for _, r in cases]
    levels = H.Batch(plans)
    ref = [o.clone() for o in levels.evaluate(TWs, nrhs)]
    levels.status()
    one = H.Batch(plans)
    one.set_one_launch(True)
    for rep in range(2):  # the second evaluation replays the captured graph
        outs = one.evaluate(TWs, nrhs)
        one.status()
        for m, o, y, want in zip(modes, outs, ref, wants):
            err = np.linalg.norm(o.cpu().numpy() - want) / np.linalg.norm(want)
            assert 1e-12 < err <= (5e-6 if m != "split_bf16" else 1e-5), (rep, m, err)
            assert torch.linalg.norm(o - y).item() <= 1e-6 * np.linalg.norm(want), (rep, m)
    assert one.info()["launches"] == 1 < levels.info()["launches"]
    recs = one.profile(TWs, nrhs, [torch.zeros_like(t) for t in TWs])
    one.status()
    assert sum(not x["chained"] for x in recs) == 1
    assert sum(x["flops"] for x in recs) == sum(c.flops(r) for c, r in cases)
    # every level's own span, from the kernel's timer, inside the launch's event time
    assert all(x["level_ms"] > 0.0 for x in recs)
    assert sum(x["level_ms"] for x in recs) <= 1.05 * recs[0]["ms"]
