"""Tree reuse on the GPU (gt_tree_events / gt_tree_refresh / gt_tree_particles): the incremental
node moments of shmem/tree.cc:211-329 and a walk on the refreshed tree, against the reference's own
results for the same events (tests/golden/reuse_scenario.py, golden ``reuse_*``).

Bars: node centre of mass, velocity and mass to 1e-12 (FP64; kicks and shifts are applied with
atomics, in another order); speed bounds, displacement pads, node softenings and sides (float)
bit-exact; opening radius 1e-12; the walk on the reused tree to the walk bars (median 1e-5).
"""
import os
import sys

import numpy as np
import pytest

import gizmo_shared_memory_b200 as g

pytestmark = pytest.mark.gpu
sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
import reuse_scenario as RS  # noqa: E402


def cell_map(nd):
    return {(int(l), float(a), float(b), float(c)): i
            for i, (l, a, b, c) in enumerate(zip(nd["level"], nd["gcx"], nd["gcy"], nd["gcz"]))}


def particles(golden):
    return {k: golden[f"plummer_{k}"] for k in ("x", "y", "z", "m", "soft")}


def test_reuse_matches_reference(gpu_ctx, oracle, golden):
    P = particles(golden)
    vel = [golden[f"plummer_v{k}"] for k in "xyz"]
    T = gpu_ctx.build(P, key_mode=g.GT_KEY_MORTON)
    gpu_ctx.tree_velocities(T, *vel)
    d = T.download()
    leaf = d["leaf_of"]
    evs = RS.events(P, vel)
    for kind, parts, arr, tau in evs:
        gpu_ctx.tree_events(T, kind, leaf[parts], a=arr.get("a"), x=arr.get("x"), v=arr.get("v"),
                            f=arr.get("f"), tau=tau)
    gpu_ctx.tree_refresh(T, RS.TAU)
    st = gpu_ctx.tree_node_state(T, RS.TAU)
    nd = T.download()
    on = oracle.build(P).nodes()  # the reference's numbering (golden arrays are indexed by it)
    gm, om = cell_map(nd), cell_map(on)
    assert gm.keys() == om.keys()
    gi = np.array([gm[k] for k in om])
    oi = np.array([om[k] for k in om])
    scale = np.abs(golden["reuse_com"]).max()
    assert np.abs(st["com"][gi] - golden["reuse_com"][oi]).max() <= 1e-12 * scale
    assert np.abs(st["vel"][gi] - golden["reuse_vel"][oi]).max() <= 1e-12 * np.abs(golden["reuse_vel"]).max()
    np.testing.assert_allclose(st["mass"][gi], golden["reuse_mass"][oi], rtol=1e-12, atol=1e-18)
    for k in ("vmax", "xpad"):
        assert np.array_equal(st[k][gi], golden[f"reuse_{k}"][oi]), k
    assert np.array_equal(nd["w_len"][gi], golden["reuse_w_len"][oi])
    assert np.array_equal(nd["w_soft"][gi], golden["reuse_w_soft"][oi])
    np.testing.assert_allclose(nd["w_s"][gi], golden["reuse_w_s"][oi], rtol=1e-12)
    # the walk node's centre of mass and mass are the refreshed ones
    assert np.abs(np.stack([nd["cx"], nd["cy"], nd["cz"]], 1)[gi] - golden["reuse_com"][oi]).max() <= 1e-12 * scale
    # the walk on the reused tree, with the particles' positions a time tau later
    x, y, z = RS.positions_after(P, vel, evs)
    gpu_ctx.tree_particles(T, x, y, z)
    tg = golden["plummer_orderbuf"]
    ax, ay, az = gpu_ctx.accel_grouped(T, tg, aold=golden["plummer_aold"])
    a = np.stack([ax, ay, az], 1)
    b = np.stack([golden["reuse_ax"], golden["reuse_ay"], golden["reuse_az"]], 1)
    e = np.linalg.norm(a - b, axis=1) / np.linalg.norm(b, axis=1)
    assert np.median(e) <= 1e-5 and np.quantile(e, 0.99) <= 2e-3, (np.median(e), np.quantile(e, 0.99))


def test_reuse_without_node_velocities(gpu_ctx, golden):
    """Without velocities the momentum events are no-ops, as in the reference (tree.cc:212, 230,
    249); the bounds still move, and refresh only widens the radii."""
    P = particles(golden)
    T = gpu_ctx.build(P)
    d0 = T.download()
    leaf = d0["leaf_of"]
    live = np.nonzero(P["m"] > 0)[0][:10]
    gpu_ctx.tree_events(T, 0, leaf[live],
                        a=np.ones((10, 3)), tau=0.1)
    gpu_ctx.tree_events(T, 5, leaf[live], a=np.full(10, 0.01))
    gpu_ctx.tree_refresh(T, 0.1)
    d1 = T.download()
    st = gpu_ctx.tree_node_state(T, 0.1)
    for k in ("cx", "cy", "cz", "mass"):
        assert np.array_equal(d1[k], d0[k]), k
    grown = d1["w_s"] - d0["w_s"]
    assert np.all(grown >= 0) and np.allclose(grown, 2.0 * st["xpad"].astype(np.float64))


def test_reuse_errors(gpu_ctx, golden):
    T = gpu_ctx.build(particles(golden))
    with pytest.raises(g.GTError) as e:
        gpu_ctx.tree_events(T, 9, np.zeros(1, np.int32), a=np.zeros(1))
    assert e.value.status == 1
    with pytest.raises(g.GTError) as e:
        gpu_ctx.tree_events(T, 0, np.array([10 ** 8], np.int32), a=np.zeros((1, 3)))
    assert e.value.status == 1


@pytest.mark.parametrize("kind", [0, 1])
def test_many_events_sum_by_level(gpu_ctx, kind):
    """A call with many kicks (kind 0) or shifts (kind 1) sums them per leaf and carries the sums up
    one tree level at a time; the same events applied in calls small enough to climb the parent
    chain per event give the same node state to 1e-12 (FP64, another summation order)."""
    from gizmo_shared_memory_b200 import ics

    P = ics.plummer(n=300000, seed=31, soft=0.01)
    rng = np.random.default_rng(6)
    vel = [rng.normal(0.0, 0.5, 300000) for _ in range(3)]
    trees = []
    for _ in range(2):
        T = gpu_ctx.build(P)
        gpu_ctx.tree_velocities(T, *vel)
        trees.append(T)
    leaf = trees[0].download(nodes=False)["leaf_of"]
    live = np.nonzero(leaf >= 0)[0]
    vec = rng.normal(0.0, 1e-3, (len(live), 3))
    tau = 0.01
    kw = dict(a=vec, tau=tau) if kind == 0 else dict(a=P["m"][live], x=vec)
    gpu_ctx.tree_events(trees[0], kind, leaf[live], **kw)  # one call: sums by level
    for s in range(0, len(live), 50000):  # small calls: per-event climbs
        part = slice(s, s + 50000)
        kw2 = dict(a=vec[part], tau=tau) if kind == 0 else dict(a=P["m"][live][part], x=vec[part])
        gpu_ctx.tree_events(trees[1], kind, leaf[live][part], **kw2)
    st = [gpu_ctx.tree_node_state(T, 0.02) for T in trees]
    for k in ("com", "vel", "mass"):
        scale = np.abs(st[1][k]).max()
        assert np.abs(st[0][k] - st[1][k]).max() <= 1e-12 * scale, k
