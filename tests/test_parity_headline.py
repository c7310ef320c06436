"""GPU parity at the sizes the throughput metric is quoted on.

The workloads are the 16M clustered box, the 4M isolated galaxy and the 67M merger (generators in
gizmo_shared_memory_b200/ics.py).  Each is walked as bench.py walks it:
  * the GPU tree (Peano-Hilbert order, 20-bit cells as shmem::build), a bootstrap walk with
    Barnes-Hut theta = 0.7 and aold = 0, aold = alpha |a| / G (shmem/mfm.cc:743-751);
  * then the relative criterion alone, windows of 32 consecutive targets in the GPU's tree order.

The checker is the reference's own shmem::accel_grouped (shmem/tree.cc:626-897), compiled from its
sources into oracle/_ref (the pinned restatement oracle/gt_oracle.c where that is absent), on its
own tree of the same particles.  It walks a random sample of whole GPU windows, passed in GPU tree
order with batch = 32, so its fixed windows (tree.cc:668-670) are exactly the GPU's windows: the
same group boxes, the same smallest aold, the same nodes offered to the criterion.  Both get the
same aold.

Bars: median relative error <= 1e-5 (FP32 interaction arithmetic on FP64 group-relative offsets);
p99 <= 2e-3, for the rare target whose group sees an opening decision flip at the threshold (the
node moments are summed in a different order).
"""
import numpy as np
import pytest

import gizmo_shared_memory_b200 as g
from gizmo_shared_memory_b200 import ics

pytestmark = pytest.mark.gpu

MEDIAN_TOL = 1e-5
P99_TOL = 2e-3
WINDOW = 32


def relerr(a, b):
    d = np.sqrt(sum((x - y) ** 2 for x, y in zip(a, b)))
    n = np.sqrt(sum(y ** 2 for y in b))
    return d / np.where(n > 0, n, 1.0)


def checker(P):
    """The compiled reference when present, else the pinned restatement; a tree of P."""
    from oracle import Reference, Restatement, reference_available

    if reference_available():
        R = Reference()
        R.set_threads(R.max_threads())
        return "reference", R.build(P)
    return "restatement", Restatement().build(P)


def walk_windows(kind, tree, targets, theta, aold):
    if kind == "reference":
        return tree.accel_grouped(targets, theta, 1.0, WINDOW, aold=aold)
    return tree.accel_grouped(targets, theta, 1.0, WINDOW, aold=aold)[:3]


def headline_parity(P, alpha, n_windows, seed):
    import torch

    ctx = g.Context(0)
    dev = {k: torch.as_tensor(v, device="cuda") for k, v in P.items()}
    T = ctx.build(dev)
    nl = T.info()["n_live"]
    ob = T.download(nodes=False)["orderbuf"]
    del dev
    out = tuple(torch.empty(nl, dtype=torch.float64, device="cuda") for _ in range(3))
    ctx.accel_grouped(T, None, theta=0.7, batch=WINDOW, outs=out + (None,), group_mode=g.GT_GROUP_BATCH)
    boot = [o.cpu().numpy() for o in out]
    aold = ctx.form_aold(*out, alpha)
    ctx.accel_grouped(T, None, aold=aold, theta=0.0, batch=WINDOW, outs=out + (None,),
                      group_mode=g.GT_GROUP_BATCH)
    walk = [o.cpu().numpy() for o in out]
    aold = aold.cpu().numpy()
    T.free()
    ctx.close()

    rng = np.random.default_rng(seed)
    w = np.sort(rng.choice(nl // WINDOW, size=n_windows, replace=False))
    pos = (w[:, None] * WINDOW + np.arange(WINDOW)[None, :]).ravel()
    kind, R = checker(P)
    rb = walk_windows(kind, R, ob[pos], 0.7, None)
    rw = walk_windows(kind, R, ob[pos], 0.0, aold[pos])
    eb = relerr([a[pos] for a in boot], rb)
    ew = relerr([a[pos] for a in walk], rw)
    return kind, len(pos), eb, ew


def report(name, kind, nt, eb, ew):
    print(f"{name}: {nt} targets in whole windows of {WINDOW}, checker {kind}: "
          f"bootstrap median {np.median(eb):.2e} p99 {np.quantile(eb, 0.99):.2e}; "
          f"relative criterion median {np.median(ew):.2e} p99 {np.quantile(ew, 0.99):.2e}")
    for e in (eb, ew):
        assert np.isfinite(e).all()
        assert np.median(e) <= MEDIAN_TOL, np.median(e)
        assert np.quantile(e, 0.99) <= P99_TOL, np.quantile(e, 0.99)


def test_parity_clustered_16m():
    P = ics.soneira_peebles(seed=3)
    report("clustered_16m", *headline_parity(P, 0.0025, 384, 11))


def test_parity_galaxy_4m():
    P = ics.galaxy(seed=2)
    report("galaxy_4m", *headline_parity(P, 0.0025, 384, 12))


def test_parity_merger_67m():
    P = ics.merger(seed=5)
    report("merger_67m", *headline_parity(P, 0.0025, 256, 13))


def test_parity_sparse_active_galaxy_4m():
    """A scattered 1 % active set in tree order -- the engine's deep-timebin steps hand the walk
    their active targets in tree order (shmem/mfm.cc:698-732) -- grouped by leaf (batch 0, the
    engine's grouping) and in windows of 32, against the reference on the same targets and aold.
    The group count of such a call stays on the device; the counted walk reports it."""
    import torch

    P = ics.galaxy(seed=2)
    ctx = g.Context(0)
    dev = {k: torch.as_tensor(v, device="cuda") for k, v in P.items()}
    T = ctx.build(dev)
    nl = T.info()["n_live"]
    ob = T.download(nodes=False)["orderbuf"]
    out = tuple(torch.empty(nl, dtype=torch.float64, device="cuda") for _ in range(3))
    ctx.accel_grouped(T, None, theta=0.7, batch=WINDOW, outs=out + (None,), group_mode=g.GT_GROUP_BATCH)
    aold = ctx.form_aold(*out, 0.0025).cpu().numpy()
    rng = np.random.default_rng(14)
    pos = np.sort(rng.choice(nl, size=nl // 100, replace=False))
    tg = ob[pos].astype(np.uint32)
    kind, R = checker(P)
    leaf = R.order()[2]
    for batch, mode in ((0, g.GT_GROUP_LEAF), (WINDOW, g.GT_GROUP_BATCH)):
        a = ctx.accel_grouped(T, tg, aold=aold[pos], batch=batch, group_mode=mode, count=True)
        st = ctx.stats()
        if batch == 0:
            lv = leaf[tg]
            assert st["groups"] == 1 + int(np.count_nonzero(lv[1:] != lv[:-1]))
        else:
            assert st["groups"] == -(-len(tg) // WINDOW)
        r = walk_windows(kind, R, tg, 0.0, aold[pos]) if batch else (
            R.accel_grouped(tg, 0.0, 1.0, 0, aold=aold[pos])[:3])
        e = relerr(a, r)
        print(f"galaxy_4m scattered 1 %: {len(tg)} targets, batch {batch}: median {np.median(e):.2e} "
              f"p99 {np.quantile(e, 0.99):.2e}")
        assert np.median(e) <= MEDIAN_TOL and np.quantile(e, 0.99) <= P99_TOL
    ctx.close()


def test_parity_tidal_jerk_galaxy_4m():
    """The tidal tensor and the jerk (shmem::accel_grouped's `tidal` and `jerk`, tree.cc:811-880)
    at full size: the 4M galaxy with seeded velocities, windows of 32 in GPU tree order, against the
    reference's own extended walk on a tree built with the same velocities (tree.cc:149-190).
    Per target, the Frobenius norm of the difference over the reference's norm: median <= 1e-5."""
    import torch
    from oracle import Reference, reference_available

    if not reference_available():
        pytest.skip("oracle/_ref not built")
    P = ics.galaxy(seed=2)
    rng = np.random.default_rng(21)
    vel = [0.1 * rng.standard_normal(len(P["m"])) for _ in range(3)]
    ctx = g.Context(0)
    dev = {k: torch.as_tensor(v, device="cuda") for k, v in P.items()}
    T = ctx.build(dev)
    ctx.tree_velocities(T, *vel)
    nl = T.info()["n_live"]
    ob = T.download(nodes=False)["orderbuf"]
    out = tuple(torch.empty(nl, dtype=torch.float64, device="cuda") for _ in range(3))
    ctx.accel_grouped(T, None, theta=0.7, batch=WINDOW, outs=out + (None,), group_mode=g.GT_GROUP_BATCH)
    aold = ctx.form_aold(*out, 0.0025).cpu().numpy()
    w = np.sort(np.random.default_rng(22).choice(nl // WINDOW, size=256, replace=False))
    pos = (w[:, None] * WINDOW + np.arange(WINDOW)[None, :]).ravel()
    tg = ob[pos].astype(np.uint32)
    ax, ay, az, _, tt, jj = ctx.accel_grouped_ext(T, tg, aold=aold[pos], batch=WINDOW, tidal=True, jerk=True,
                                                  group_mode=g.GT_GROUP_BATCH)
    ctx.close()
    R = Reference()
    R.set_threads(R.max_threads())
    RT = R.build(P, vel=vel)
    rx, ry, rz, rt, rj = RT.accel_grouped_ext(tg, 0.0, 1.0, WINDOW, aold=aold[pos], tidal=True, jerk=True)
    ea = relerr((ax, ay, az), (rx, ry, rz))
    et = np.linalg.norm(tt - rt, axis=1) / np.linalg.norm(rt, axis=1)
    ej = np.linalg.norm(jj - rj, axis=1) / np.linalg.norm(rj, axis=1)
    print(f"galaxy_4m tidal/jerk, {len(tg)} targets: acceleration median {np.median(ea):.2e}; tidal median "
          f"{np.median(et):.2e} p99 {np.quantile(et, 0.99):.2e}; jerk median {np.median(ej):.2e} "
          f"p99 {np.quantile(ej, 0.99):.2e}")
    for e in (ea, et, ej):
        assert np.isfinite(e).all()
        assert np.median(e) <= MEDIAN_TOL and np.quantile(e, 0.99) <= P99_TOL
