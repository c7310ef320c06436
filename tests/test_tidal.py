"""Tidal tensor and jerk in the GPU walk (shmem::accel_grouped's `tidal` and `jerk`,
shmem/tree.cc:811-880), and the per-node velocity moments they need (tree.cc:149-190).

Bars: node centre-of-mass velocities to 1e-12 (FP64, another summation order), speed bounds
bit-exact; tidal tensor and jerk from FP32 interaction arithmetic on FP64 group-relative offsets,
so per target the relative error (Frobenius norm of the difference over the reference's norm)
has a median <= 1e-5 and a p99 <= 2e-3 against the reference's own values (golden fixtures) and
the oracle restatement.
"""
import numpy as np
import pytest

import gizmo_shared_memory_b200 as g

pytestmark = pytest.mark.gpu


def particles(golden):
    return {k: golden[f"plummer_{k}"] for k in ("x", "y", "z", "m", "soft")}


def cell_map(nd):
    return {(int(l), float(a), float(b), float(c)): i
            for i, (l, a, b, c) in enumerate(zip(nd["level"], nd["gcx"], nd["gcy"], nd["gcz"]))}


def rel_rows(a, b):
    return np.linalg.norm(a - b, axis=1) / np.linalg.norm(b, axis=1)


@pytest.fixture(scope="module")
def vtree(gpu_ctx, golden):
    P = particles(golden)
    vel = [golden[f"plummer_v{k}"] for k in "xyz"]
    T = gpu_ctx.build(P, key_mode=g.GT_KEY_MORTON)
    gpu_ctx.tree_velocities(T, *vel)
    return P, vel, T


def test_velocity_moments_match_reference(gpu_ctx, oracle, golden, vtree):
    P, vel, T = vtree
    vg, vmg = gpu_ctx.velocity_moments(T)
    gn = T.download()
    on = oracle.build(P).nodes()
    gm, om = cell_map(gn), cell_map(on)
    assert gm.keys() == om.keys()
    gi = np.array([gm[k] for k in om])
    oi = np.array([om[k] for k in om])
    for k, v in zip("xyz", vg):
        ref = golden[f"plummer_vcom_{k}"][oi]
        assert np.all(np.abs(v[gi] - ref) <= 1e-12 * (np.abs(ref) + 1.0)), k
    assert np.array_equal(vmg[gi], golden["plummer_vmax"][oi])


@pytest.mark.parametrize("name,theta,batch", [("bh", 0.7, 0), ("b8", 0.7, 8), ("rel", 0.0, 0)])
def test_tidal_and_jerk_match_reference(gpu_ctx, golden, vtree, name, theta, batch):
    P, vel, T = vtree
    tg = golden["plummer_orderbuf"]
    aold = golden["plummer_aold"] if name == "rel" else None
    ax, ay, az, _, tt, jj = gpu_ctx.accel_grouped_ext(T, tg, aold=aold, theta=theta, batch=batch, tidal=True,
                                                      jerk=True)
    gt, gj = golden[f"plummer_{name}_tidal"], golden[f"plummer_{name}_jerk"]
    et, ej = rel_rows(tt, gt), rel_rows(jj, gj)
    assert np.median(et) <= 1e-5 and np.quantile(et, 0.99) <= 2e-3, (np.median(et), np.quantile(et, 0.99))
    assert np.median(ej) <= 1e-5 and np.quantile(ej, 0.99) <= 2e-3, (np.median(ej), np.quantile(ej, 0.99))
    # the accelerations of the extended walk are those of the plain one
    bx, by, bz = gpu_ctx.accel_grouped(T, tg, aold=aold, theta=theta, batch=batch)
    a = np.stack([ax, ay, az], 1)
    b = np.stack([bx, by, bz], 1)
    assert np.median(rel_rows(a, b)) < 1e-6


def test_tidal_only_and_all_live(gpu_ctx, oracle, golden, vtree):
    """Tidal tensor without the jerk (no velocities read), every live particle as target, in
    both output orders, with the potential from the same walk."""
    P, vel, T = vtree
    O = oracle.build(P)
    ob = golden["plummer_orderbuf"]
    starts = O.groups(ob, 0)
    _, _, _, ot, _ = O.walk_groups_ext(ob, starts, 0.7)
    _, _, _, phi, tt, jj = gpu_ctx.accel_grouped_ext(T, None, theta=0.7, tidal=True, jerk=False, want_phi=True)
    assert jj is None
    et = rel_rows(tt, ot)  # tree order == the oracle's orderbuf order (Morton keys)
    assert np.median(et) <= 1e-5 and np.quantile(et, 0.99) <= 2e-3
    _, _, _, _, to, _ = gpu_ctx.accel_grouped_ext(T, None, theta=0.7, tidal=True, out_order=g.GT_OUT_ORIGINAL)
    assert np.array_equal(to[ob], tt)
    massless = P["m"] <= 0
    assert np.all(to[massless] == 0)
    phi_ref = gpu_ctx.accel_grouped(T, None, theta=0.7, want_phi=True)[3]
    np.testing.assert_allclose(phi, phi_ref, rtol=1e-6)


def test_tidal_errors(gpu_ctx, golden):
    P = particles(golden)
    T = gpu_ctx.build(P)
    with pytest.raises(g.GTError) as e:  # the jerk needs velocities
        gpu_ctx.accel_grouped_ext(T, None, theta=0.7, tidal=False, jerk=True)
    assert e.value.status == 1
    model = np.zeros(g._gt.MAC_MODEL_FLOATS, np.float32)
    model[8:16] = 1.0
    with pytest.raises(g.GTError) as e:  # plain criterion only
        gpu_ctx.accel_grouped_ext(T, None, aold=np.full(T.info()["n_live"], 1e-3), tidal=True,
                                  mac_model=model, mac_kappa=1.0, mac_band=(0.01, 100.0))
    assert e.value.status == 4
    with pytest.raises(g.GTError) as e:
        gpu_ctx.accel_grouped_ext(T, None, theta=0.7, tidal=True, list_capacity=1024)
    assert e.value.status == 1
    # the context stays usable
    assert gpu_ctx.accel_grouped_ext(T, None, theta=0.7, tidal=True)[4].shape == (T.info()["n_live"], 6)
