"""Walk plans (the all-active walk captured as a CUDA graph), interaction-list capacity as a launch
parameter, and the autotuner.

  * a plan replays exactly the walk gt_accel_grouped makes (bit-identical), picks up new aold
    contents between launches, and walks every system of a forest in one replay;
  * list capacities 64..1024 change only where the lists are flushed: results agree with the
    default to FP32 summation-order level;
  * the autotuner returns a configuration whose sampled p99 meets the target and that is the
    fastest accepted candidate it measured; with a model it also measures the learned criterion.
"""
import numpy as np
import pytest

import gizmo_shared_memory_b200 as g
from gizmo_shared_memory_b200 import ics

pytestmark = pytest.mark.gpu


def host(xs):
    return np.stack([x.cpu().numpy() if hasattr(x, "cpu") else np.asarray(x) for x in xs])


@pytest.fixture(scope="module")
def setup():
    import torch

    ctx = g.Context(0, torch_stream=True)
    P = ics.plummer(n=65536, seed=42, soft=0.01)
    T = ctx.build(P)
    nl = T.info()["n_live"]
    outs = tuple(torch.empty(nl, dtype=torch.float64, device="cuda") for _ in range(3))
    ctx.accel_grouped(T, None, theta=0.7, outs=outs + (None,), group_mode=g.GT_GROUP_BATCH, batch=32)
    aold = ctx.form_aold(*outs, 0.005)
    return ctx, P, T, aold


def test_plan_replays_the_walk(setup):
    import torch

    ctx, P, T, aold = setup
    nl = T.info()["n_live"]
    kw = dict(group_mode=g.GT_GROUP_BATCH, batch=32)
    want = host(ctx.accel_grouped(T, None, aold=aold, **kw))
    outs = tuple(torch.zeros(nl, dtype=torch.float64, device="cuda") for _ in range(3))
    a2 = aold.clone()
    plan = ctx.plan(T, a2, outs, **kw)
    for o in outs:
        o.zero_()
    plan.launch()
    plan.launch()
    torch.cuda.synchronize()
    assert np.array_equal(host(outs), want)
    # new aold contents, same addresses
    a2.mul_(3.0)
    plan.launch()
    torch.cuda.synchronize()
    want3 = host(ctx.accel_grouped(T, None, aold=a2, **kw))
    assert np.array_equal(host(outs), want3)
    assert not np.array_equal(want3, want)
    plan.free()


def test_plan_on_a_forest(setup):
    import torch

    ctx = setup[0]
    P, off, _ = ics.plummer_batch(n_systems=16, n_min=300, n_max=30000, n_total=100000, seed=9, spacing=50.0)
    F = ctx.build(P, offsets=off)
    nl = F.info()["n_live"]
    outs = tuple(torch.zeros(nl, dtype=torch.float64, device="cuda") for _ in range(3))
    aold = torch.zeros(nl, dtype=torch.float64, device="cuda")
    plan = ctx.plan(F, aold, outs, theta=0.6, group_mode=g.GT_GROUP_BATCH, batch=32)
    plan.launch()
    torch.cuda.synchronize()
    want = host(ctx.accel_grouped(F, None, theta=0.6, group_mode=g.GT_GROUP_BATCH, batch=32))
    assert np.array_equal(host(outs), want)
    plan.free()


@pytest.mark.parametrize("cap", [64, 128, 512, 1024])
def test_list_capacity(setup, cap):
    ctx, P, T, aold = setup
    kw = dict(group_mode=g.GT_GROUP_BATCH, batch=32, aold=aold)
    ref = host(ctx.accel_grouped(T, None, **kw))
    got = host(ctx.accel_grouped(T, None, list_capacity=cap, **kw))
    d = np.linalg.norm(got - ref, axis=0) / np.linalg.norm(ref, axis=0)
    assert np.median(d) < 1e-6 and d.max() < 1e-4
    for warps in (2, 4):
        got = host(ctx.accel_grouped(T, None, list_capacity=cap, block_warps=warps, **kw))
        d = np.linalg.norm(got - ref, axis=0) / np.linalg.norm(ref, axis=0)
        assert np.median(d) < 1e-6


def test_list_capacity_invalid(setup):
    ctx, P, T, aold = setup
    with pytest.raises(g.GTError) as e:
        ctx.accel_grouped(T, None, aold=aold, group_mode=g.GT_GROUP_BATCH, batch=32, list_capacity=100)
    assert e.value.status == 1


def test_autotune_meets_target(setup):
    ctx, P, T, aold = setup
    rng = np.random.default_rng(5)
    sample = np.sort(rng.choice(len(P["m"]), 512, replace=False)).astype(np.uint32)
    ref = ctx.direct(P, sample, want_phi=False)[:3]
    target = 1e-2
    opts, entries = ctx.autotune(T, aold, sample=sample, ref=ref, p99_max=target, reps=2)
    assert len(entries) >= 7
    acc = [e for e in entries if e["accepted"]]
    assert acc, entries
    fastest = min(acc, key=lambda e: e["ms"])
    assert opts["block_warps"] == fastest["block_warps"]
    assert opts["list_capacity"] == fastest["list_capacity"]
    # the chosen configuration, run through the ordinary call, gives the error the tuner measured
    kw = {k: v for k, v in opts.items() if k != "batch"}
    full = ctx.accel_grouped(T, None, aold=aold, batch=opts["batch"], out_order=g.GT_OUT_ORIGINAL, **kw)
    got = host(full)[:, sample]
    e = np.linalg.norm(got - np.stack(ref), axis=0) / np.linalg.norm(np.stack(ref), axis=0)
    assert np.quantile(e, 0.99) == pytest.approx(fastest["p99"], rel=1e-9)
    assert np.quantile(e, 0.99) <= target


def test_autotune_tries_the_learned_criterion(setup):
    ctx, P, T, aold = setup
    # the zero network reproduces the plain criterion at kappa = 1
    model = np.zeros(g._gt.MAC_MODEL_FLOATS, np.float32)
    model[8:16] = 1.0
    opts, entries = ctx.autotune(T, aold, reps=1, mac_model=model, kappas=[1.0, 2.0], mac_band=(0.01, 100.0))
    learned = [e for e in entries if e["mac"] == g.GT_MAC_LEARNED]
    assert len(learned) == 2
    assert all(e["mac_kappa"] in (1.0, 2.0) for e in learned)
