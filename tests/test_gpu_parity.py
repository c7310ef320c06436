"""GPU parity: the sm_100a path, called through the C ABI, against the oracle and the fixtures.

Bars (stated per test):
  * keys, sort order, tree topology, leaf membership: bit-exact (integer work);
  * node moments: FP64, relative 1e-12 (the GPU reduces in a different summation order);
  * walks: FP32 interaction arithmetic on FP64 group-relative offsets, so the acceleration must match
    the oracle walk with the same opening criterion to a median relative error <= 1e-5; p99 is
    bounded loosely (a few targets may see an opening decision flip at the threshold);
  * FP64 direct sum: relative 1e-12.
"""
import numpy as np
import pytest

import gizmo_shared_memory_b200 as g
from gizmo_shared_memory_b200 import ics

pytestmark = pytest.mark.gpu

MEDIAN_TOL = 1e-5


def relerr(ax, ay, az, bx, by, bz):
    d = np.sqrt((ax - bx) ** 2 + (ay - by) ** 2 + (az - bz) ** 2)
    n = np.sqrt(bx ** 2 + by ** 2 + bz ** 2)
    return d / np.where(n > 0, n, 1.0)


def stable_order(keys, m):
    live = np.nonzero(m > 0)[0]
    return live[np.argsort(keys[live], kind="stable")].astype(np.uint32)


@pytest.fixture(scope="module")
def plummer():
    return ics.plummer(n=65536, seed=42, soft=0.01)


@pytest.fixture(scope="module")
def plummer_trees(gpu_ctx, oracle, plummer):
    return gpu_ctx.build(plummer, key_mode=g.GT_KEY_MORTON), oracle.build(plummer)


# ---- keys and sort --------------------------------------------------------------------------

@pytest.mark.parametrize("mode", [g.GT_KEY_MORTON, g.GT_KEY_PEANO])
def test_keys_and_order_bit_exact(gpu_ctx, oracle, plummer, mode):
    P = dict(plummer)
    P["m"] = P["m"].copy()
    P["m"][::101] = 0.0  # massless particles sort last and stay out of the tree
    T = gpu_ctx.build(P, key_mode=mode)
    keys, _ = oracle.keys20(P, key_mode=0 if mode == g.GT_KEY_MORTON else 1)
    want = stable_order(keys, P["m"])
    d = T.download(nodes=False)
    assert np.array_equal(d["orderbuf"], want)
    assert np.array_equal(T.keys(), keys[want])
    rank = np.full(len(P["m"]), np.iinfo(np.uint32).max, np.uint32)
    rank[want] = np.arange(len(want), dtype=np.uint32)
    assert np.array_equal(d["rank"], rank)


def test_peano_keys_42bit_golden(gpu_ctx, golden):
    for bits in (1, 2, 3, 20, 42):
        xyz = golden[f"keys{bits}_xyz"].astype(np.float64)
        pos = xyz * 2.0 ** -bits  # (pos - 0)/1 + 1 has exactly these top mantissa bits
        ph_hi, ph_lo, mo_hi, mo_lo = gpu_ctx.peano_keys(pos[:, 0], pos[:, 1], pos[:, 2], (0, 0, 0), 1.0, bits)
        if bits <= 3:
            assert np.array_equal(ph_lo, golden[f"keys{bits}_ph"])
            assert np.array_equal(mo_lo, golden[f"keys{bits}_morton"])
        else:
            assert np.array_equal(ph_hi, golden[f"keys{bits}_ph_hi"])
            assert np.array_equal(ph_lo, golden[f"keys{bits}_ph_lo"])
            assert np.array_equal(mo_hi, golden[f"keys{bits}_morton_hi"])
            assert np.array_equal(mo_lo, golden[f"keys{bits}_morton_lo"])


def test_peano_keys_42bit_random(gpu_ctx, oracle):
    rng = np.random.default_rng(9)
    x, y, z = rng.uniform(-3, 5, (3, 5000))
    corner, length = (-3.5, -3.5, -3.5), 9.0
    ph_hi, ph_lo, _, _ = gpu_ctx.peano_keys(x, y, z, corner, length, 42)
    for k in range(0, 5000, 7):
        xb = oracle.double_to_int((x[k] - corner[0]) / length + 1.0, 42)
        yb = oracle.double_to_int((y[k] - corner[1]) / length + 1.0, 42)
        zb = oracle.double_to_int((z[k] - corner[2]) / length + 1.0, 42)
        key = oracle.peano_key(xb, yb, zb, 42)
        assert (int(ph_hi[k]) << 64) | int(ph_lo[k]) == key


# ---- tree -----------------------------------------------------------------------------------

def cell_map(nd):
    return {(int(l), float(a), float(b), float(c)): i
            for i, (l, a, b, c) in enumerate(zip(nd["level"], nd["gcx"], nd["gcy"], nd["gcz"]))}


@pytest.mark.parametrize("mode", [g.GT_KEY_MORTON, g.GT_KEY_PEANO])
def test_tree_matches_oracle(gpu_ctx, oracle, plummer, mode):
    T = gpu_ctx.build(plummer, key_mode=mode)
    O = oracle.build(plummer)
    gn, on = T.download(), O.nodes()
    assert len(gn["mass"]) == len(on["mass"])
    gm, om = cell_map(gn), cell_map(on)
    assert gm.keys() == om.keys()  # the same cells, bit-exact centres and levels
    gi = np.array([gm[k] for k in om])
    oi = np.array([om[k] for k in om])
    for k in ("size", "w_len", "w_soft", "soft"):
        assert np.array_equal(gn[k][gi], on[k][oi]), k
    np.testing.assert_allclose(gn["mass"][gi], on["mass"][oi], rtol=1e-12)
    scale = on["size"][oi]
    for k in ("cx", "cy", "cz"):
        assert np.all(np.abs(gn[k][gi] - on[k][oi]) <= 1e-12 * scale), k
    assert np.all(np.abs(gn["w_s"][gi] - on["w_s"][oi]) <= 1e-12 * scale)
    assert np.array_equal(gn["phi"][gi] - gn["plo"][gi], on["phi"][oi] - on["plo"][oi])
    assert np.array_equal(gn["first"][gi] < 0, on["first"][oi] < 0)
    # leaf membership is the same set of particles per cell
    gob, oob = gn["orderbuf"], O.order()[0]
    leaves = np.nonzero(on["first"][oi] < 0)[0]
    for j in leaves[:: max(1, len(leaves) // 500)]:
        a, b = gi[j], oi[j]
        assert set(gob[gn["plo"][a]:gn["phi"][a]]) == set(oob[on["plo"][b]:on["phi"][b]])
    if mode == g.GT_KEY_MORTON:
        assert np.array_equal(gob, oob)


def test_tree_threading_audit(gpu_ctx, plummer):
    """The reference's audit (tree.cc:986-1015): next-chain children, every particle reached once."""
    T = gpu_ctx.build(plummer)
    d = T.download()
    first, nxt, parent = d["first"], d["next"], d["parent"]
    seen = np.zeros(len(plummer["m"]), np.int32)
    stack = [0]
    assert parent[0] == -1 and nxt[0] == -1
    visited = 0
    while stack:
        X = stack.pop()
        visited += 1
        if first[X] < 0:
            seen[d["orderbuf"][d["plo"][X]:d["phi"][X]]] += 1
            assert np.all(d["leaf_of"][d["orderbuf"][d["plo"][X]:d["phi"][X]]] == X)
            continue
        c = first[X]
        steps = 0
        while c != nxt[X]:
            assert parent[c] == X
            stack.append(c)
            c = nxt[c]
            steps += 1
            assert steps <= 8
    assert visited == len(first)
    assert np.all(seen == 1)


# ---- walks ----------------------------------------------------------------------------------

def check(a, b, tol=MEDIAN_TOL, p99=2e-3):
    e = relerr(*a, *b)
    assert np.isfinite(e).all()
    assert np.median(e) <= tol, np.median(e)
    assert np.quantile(e, 0.99) <= p99, np.quantile(e, 0.99)
    return e


def test_grouped_walk_plummer_65k(gpu_ctx, plummer_trees):
    T, O = plummer_trees
    ob = O.order()[0]
    # first walk: Barnes-Hut theta = 0.7 with aold = 0 (the bootstrap)
    ax, ay, az = gpu_ctx.accel_grouped(T, ob, theta=0.7)
    ox, oy, oz, _ = O.accel_grouped(ob, 0.7)
    check((ax, ay, az), (ox, oy, oz))
    # then the relative criterion alone with aold = alpha |a| from the oracle's first walk
    aold = 0.005 * np.sqrt(ox ** 2 + oy ** 2 + oz ** 2)
    ax, ay, az = gpu_ctx.accel_grouped(T, ob, aold=aold, theta=0.0)
    ox, oy, oz, _ = O.accel_grouped(ob, 0.0, aold=aold)
    check((ax, ay, az), (ox, oy, oz))


def test_grouped_walk_all_targets_null(gpu_ctx, plummer_trees):
    """targets == NULL walks every live particle in tree order (= targets = orderbuf)."""
    T, O = plummer_trees
    ob = O.order()[0]
    a = gpu_ctx.accel_grouped(T, None, theta=0.7)
    b = gpu_ctx.accel_grouped(T, ob, theta=0.7)
    for u, v in zip(a, b):
        assert np.array_equal(u, v)
    c = gpu_ctx.accel_grouped(T, None, theta=0.7, out_order=g.GT_OUT_ORIGINAL)
    for u, v in zip(c, a):
        assert np.array_equal(u[ob], v)


def test_grouped_walk_golden(gpu_ctx, golden):
    P = {k: golden[f"plummer_{k}"] for k in ("x", "y", "z", "m", "soft")}
    T = gpu_ctx.build(P, key_mode=g.GT_KEY_MORTON)
    tg = golden["plummer_orderbuf"]
    ref = lambda p: (golden[f"plummer_{p}_ax"], golden[f"plummer_{p}_ay"], golden[f"plummer_{p}_az"])
    check(gpu_ctx.accel_grouped(T, tg, theta=0.7), ref("bh"))
    check(gpu_ctx.accel_grouped(T, tg, theta=0.0, aold=golden["plummer_aold"]), ref("rel"))
    check(gpu_ctx.accel_grouped(T, tg, theta=0.7, batch=8), ref("b8"))
    sub = golden["plummer_sub"]
    check(gpu_ctx.accel(T, sub, theta=0.5), ref("acc"))
    phi = gpu_ctx.potential(T, sub, theta=0.5)
    e = np.abs(phi - golden["plummer_phi"]) / np.abs(golden["plummer_phi"])
    assert np.median(e) <= MEDIAN_TOL
    d = gpu_ctx.direct(P, sub)
    e = relerr(*d[:3], *ref("direct"))
    assert e.max() <= 1e-12


def test_grouped_walk_peano_tree_same_forces(gpu_ctx, plummer, plummer_trees):
    """PH and Morton trees hold the same cells: forces agree up to summation order."""
    Tm, O = plummer_trees
    Tp = gpu_ctx.build(plummer, key_mode=g.GT_KEY_PEANO)
    ob = O.order()[0]
    a = gpu_ctx.accel_grouped(Tp, ob, theta=0.7)
    b = gpu_ctx.accel_grouped(Tm, ob, theta=0.7)
    check(a, b, tol=1e-6, p99=1e-4)


def test_batch_windows_and_per_target(gpu_ctx, plummer_trees):
    T, O = plummer_trees
    ob = O.order()[0]
    check(gpu_ctx.accel_grouped(T, ob, theta=0.7, batch=8), O.accel_grouped(ob, 0.7, batch=8)[:3])
    sub = ob[::17].copy()
    check(gpu_ctx.accel(T, sub, theta=0.5), O.accel(sub, 0.5))
    phi = gpu_ctx.potential(T, sub, theta=0.5)
    ophi = O.potential(sub, 0.5)
    e = np.abs(phi - ophi) / np.abs(ophi)
    assert np.median(e) <= MEDIAN_TOL


def test_grouped_potential_matches_oracle(gpu_ctx, plummer_trees):
    T, O = plummer_trees
    ob = O.order()[0]
    ax, ay, az, phi = gpu_ctx.accel_grouped(T, ob, theta=0.7, want_phi=True)
    starts = O.groups(ob, 0)
    ox, oy, oz, ophi, _ = O.walk_groups(ob, starts, 0.7, want_phi=True)
    check((ax, ay, az), (ox, oy, oz))
    e = np.abs(phi - ophi) / np.abs(ophi)
    assert np.median(e) <= MEDIAN_TOL


@pytest.mark.parametrize("pairs", [True, False])
def test_packed_particle_lists_match_oracle(gpu_ctx, oracle, pairs):
    """Windows of 32 evaluate their particle lists two entries per packed FP32x2 instruction; a
    pair holding an entry inside the softening kernel takes the one-entry spline for both, and
    r = 0 (each target's own entry) contributes nothing on either path.  Softenings drawn from
    0.02-0.2 around a central spacing of about 0.05 put many pairs in that mixed case, with the
    two entries' kernel radii max(h_target, h_source) differing.  Accelerations and potentials
    against the oracle's windows of 32: two windows per warp and one."""
    P = ics.plummer(n=32768, seed=77)
    P["soft"] = np.random.default_rng(78).uniform(0.02, 0.2, len(P["m"]))
    T, O = gpu_ctx.build(P, key_mode=g.GT_KEY_MORTON), oracle.build(P)
    ob = O.order()[0]
    n = len(ob)
    starts = np.concatenate([np.arange(0, n, 32), [n]]).astype(np.int64)
    bx, by, bz, _, _ = O.walk_groups(ob, starts, 0.7)
    aold = 0.0025 * np.sqrt(bx ** 2 + by ** 2 + bz ** 2)
    ax, ay, az, phi = gpu_ctx.accel_grouped(T, ob, aold=aold, theta=0.0, want_phi=True, batch=32,
                                            group_mode=g.GT_GROUP_BATCH, window_pairs=pairs)
    rx, ry, rz, rphi, _ = O.walk_groups(ob, starts, 0.0, aold=aold, want_phi=True)
    check((ax, ay, az), (rx, ry, rz))
    e = np.abs(phi - rphi) / np.abs(rphi)
    assert np.median(e) <= MEDIAN_TOL and np.quantile(e, 0.99) <= 1e-4, (np.median(e), np.quantile(e, 0.99))


def node_group_starts(O, gmax):
    """Group starts of GT_GROUP_NODE over the full tree order, from the oracle tree."""
    nd = O.nodes()
    cnt = nd["phi"] - nd["plo"]
    par = nd["parent"]
    pc = np.where(par >= 0, cnt[np.maximum(par, 0)], np.iinfo(np.int32).max)
    mark = ((cnt <= gmax) & (pc > gmax)) | ((nd["first"] < 0) & (cnt > gmax))
    mark &= cnt > 0
    s = np.sort(nd["plo"][mark]).astype(np.int64)
    return np.concatenate([s, [O.nlive]])


@pytest.mark.parametrize("batch", [32, 64, 128])
def test_wide_windows_match_oracle(gpu_ctx, plummer_trees, batch):
    """Fixed windows of 32/64/128 consecutive targets: 1, 2 and 4 targets per lane."""
    T, O = plummer_trees
    ob = O.order()[0]
    aold = 0.0025 * np.ones(len(ob))
    a = gpu_ctx.accel_grouped(T, ob, aold=aold, batch=batch)
    b = O.accel_grouped(ob, 0.0, batch=batch, aold=aold)[:3]
    check(a, b)


@pytest.mark.parametrize("gmax", [16, 32, 64, 128])
def test_node_groups_match_oracle(gpu_ctx, plummer_trees, gmax):
    T, O = plummer_trees
    ob = O.order()[0]
    starts = node_group_starts(O, gmax)
    # chunks of at most the kernel's capacity, as the library splits them
    kmax = 32 if gmax <= 32 else (64 if gmax <= 64 else 128)
    ch = [starts[0]]
    for a, b in zip(starts[:-1], starts[1:]):
        x = a
        while x < b:
            x = min(x + kmax, b)
            ch.append(x)
    ch = np.array(ch, np.int64)
    aold = 0.0025 * np.ones(len(ob))
    a = gpu_ctx.accel_grouped(T, None, aold=aold, group_mode=g.GT_GROUP_NODE, group_max=gmax)
    b = O.walk_groups(ob, ch, 0.0, aold=aold)[:3]
    check(a, b)


def test_interaction_counts_match_oracle(gpu_ctx, plummer_trees):
    T, O = plummer_trees
    ob = O.order()[0]
    gpu_ctx.accel_grouped(T, ob, theta=0.7, count=True)
    s = gpu_ctx.stats()
    _, _, _, cnt = O.accel_grouped(ob, 0.7)
    assert s["nodes_visited"] == pytest.approx(cnt[0], rel=1e-4)
    assert s["multipole"] == pytest.approx(cnt[1], rel=1e-4)
    assert s["pairs"] == pytest.approx(cnt[2], rel=1e-4)
    assert s["groups"] == len(O.groups(ob, 0)) - 1


# ---- direct sum -----------------------------------------------------------------------------

def test_direct_fp64_and_fp32(gpu_ctx, oracle, plummer):
    tg = np.arange(0, 65536, 16, dtype=np.uint32)
    ox, oy, oz, ophi = oracle.direct(plummer, tg)
    ax, ay, az, phi = gpu_ctx.direct(plummer, tg)
    assert relerr(ax, ay, az, ox, oy, oz).max() <= 1e-12
    np.testing.assert_allclose(phi, ophi, rtol=1e-12)
    fx, fy, fz, fphi = gpu_ctx.direct(plummer, tg, precision=g.GT_DIRECT_FP32)
    e = relerr(fx, fy, fz, ox, oy, oz)
    assert np.median(e) <= 1e-5 and e.max() <= 1e-3


# ---- edge cases -----------------------------------------------------------------------------

def test_empty_single_and_pair(gpu_ctx, oracle):
    for n in (0, 1, 2, 17):
        P = ics.plummer(n=n, seed=1) if n else {k: np.zeros(0) for k in ("x", "y", "z", "m", "soft")}
        T = gpu_ctx.build(P)
        info = T.info()
        assert info["n_nodes"] >= 1 and info["n_live"] == n
        if n == 0:
            ax, ay, az = gpu_ctx.accel_grouped(T, None, theta=0.7)
            assert len(ax) == 0
            continue
        O = oracle.build(P)
        ob = O.order()[0]
        a = gpu_ctx.accel_grouped(T, ob, theta=0.7)
        b = O.accel_grouped(ob, 0.7)[:3]
        if n == 1:
            assert np.all(a[0] == 0) and np.all(a[1] == 0) and np.all(a[2] == 0)
        else:
            assert relerr(*a, *b).max() <= 1e-5


def test_collocated_level20_leaf(gpu_ctx, golden):
    Q = {k: golden[f"colloc_{k}"] for k in ("x", "y", "z", "m", "soft")}
    T = gpu_ctx.build(Q, key_mode=g.GT_KEY_MORTON)
    assert T.info()["n_nodes"] == int(golden["colloc_nnodes"][0])
    tg = golden["colloc_orderbuf"]
    a = gpu_ctx.accel_grouped(T, tg, theta=0.7)
    e = relerr(*a, golden["colloc_ax"], golden["colloc_ay"], golden["colloc_az"])
    assert np.median(e) <= MEDIAN_TOL and np.isfinite(e).all()


def test_ragged_subset_and_massless_targets(gpu_ctx, oracle, plummer):
    P = dict(plummer)
    P["m"] = P["m"].copy()
    P["m"][5::211] = 0.0
    T = gpu_ctx.build(P, key_mode=g.GT_KEY_MORTON)
    O = oracle.build(P)
    _, rank, leaf = O.order()
    rng = np.random.default_rng(4)
    act = rng.choice(len(P["m"]), 3000, replace=False).astype(np.uint32)
    live = act[rank[act] != np.iinfo(np.uint32).max]
    dead = act[rank[act] == np.iinfo(np.uint32).max]
    # active set in tree order (mfm.cc:705-711), massless targets appended: each its own group
    tg = np.concatenate([live[np.argsort(rank[live])], dead]).astype(np.uint32)
    a = gpu_ctx.accel_grouped(T, tg, theta=0.7)
    b = O.accel_grouped(tg, 0.7)[:3]
    check(a, b)


def test_host_and_device_paths_identical(gpu_ctx, plummer):
    import torch

    ctx = g.Context(0, torch_stream=True)
    T = ctx.build(plummer)
    dev = {k: torch.as_tensor(v, device="cuda") for k, v in plummer.items()}
    Td = ctx.build(dev)
    a = ctx.accel_grouped(T, None, theta=0.7)
    b = ctx.accel_grouped(Td, None, theta=0.7, device_out=True)
    for u, v in zip(a, b):
        assert np.array_equal(u, v.cpu().numpy())


def test_form_aold(gpu_ctx):
    rng = np.random.default_rng(3)
    ax, ay, az = rng.normal(size=(3, 1000))
    aold = gpu_ctx.form_aold(ax, ay, az, 0.005, G=2.0)
    np.testing.assert_allclose(aold, 0.005 * np.sqrt(ax ** 2 + ay ** 2 + az ** 2) / 2.0, rtol=1e-15)


def test_errors_leave_context_usable(gpu_ctx, plummer):
    P = dict(plummer)
    P["x"] = P["x"].copy()
    P["x"][3] = np.nan
    with pytest.raises(g.GTError) as e:
        gpu_ctx.build(P)
    assert e.value.status == 7  # GT_ERR_NONFINITE
    T = gpu_ctx.build(plummer)
    with pytest.raises(g.GTError) as e:
        gpu_ctx.accel_grouped(T, np.array([10 ** 7], np.uint32), theta=0.7)
    assert e.value.status == 1  # GT_ERR_INVALID
    # target indices are checked on the device while the walk groups them: a bad index in a long
    # list (the multi-kernel grouping), from host and from device arrays, reads nothing out of
    # bounds and fails the synchronising call
    import torch

    long = np.arange(20000, dtype=np.uint32)
    long[12345] = len(P["m"]) + 3
    with pytest.raises(g.GTError) as e:
        gpu_ctx.accel_grouped(T, long, theta=0.7)
    assert e.value.status == 1
    with pytest.raises(g.GTError) as e:
        gpu_ctx.accel_grouped(T, torch.as_tensor(long.view(np.int32), device="cuda"), theta=0.7, batch=32,
                              group_mode=g.GT_GROUP_BATCH)
    assert e.value.status == 1
    with pytest.raises(g.GTError) as e:
        gpu_ctx.accel_grouped(T, None, theta=0.7, mac=g.GT_MAC_LEARNED)
    assert e.value.status == 1  # GT_ERR_INVALID: the learned criterion without a model
    a = gpu_ctx.accel_grouped(T, None, theta=0.7)
    assert np.isfinite(a[0]).all()


def test_nonfinite_softening_rejected(gpu_ctx, plummer):
    """A build from host arrays uploads the softenings while the bounding box, keys and sort run
    and checks them in the gather stage; a non-finite softening is still GT_ERR_NONFINITE, with the
    same count as a device build gives, and the context stays usable (the next build matches one
    from device arrays bit for bit)."""
    import torch

    for bad in (np.nan, np.inf):
        P = dict(plummer)
        P["soft"] = P["soft"].copy()
        P["soft"][[5, 77]] = bad
        with pytest.raises(g.GTError) as e:
            gpu_ctx.build(P)
        assert e.value.status == 7
        assert "2 particle(s)" in str(e.value)
        dev = {k: torch.as_tensor(v, device="cuda") for k, v in P.items()}
        with pytest.raises(g.GTError) as e:
            gpu_ctx.build(dev)
        assert e.value.status == 7
        assert "2 particle(s)" in str(e.value)
    T = gpu_ctx.build(plummer)
    Td = gpu_ctx.build({k: torch.as_tensor(v, device="cuda") for k, v in plummer.items()})
    a = gpu_ctx.accel_grouped(T, None, theta=0.7)
    b = gpu_ctx.accel_grouped(Td, None, theta=0.7)
    for u, v in zip(a, b):
        assert np.array_equal(u, v)


# ---- size-independent properties at a large size ----------------------------------------------

def test_properties_galaxy_4m(gpu_ctx):
    """Full 4M-particle galaxy: G-linearity and mass scaling are exact; permuting the input leaves
    the tree order, and hence every force, bit-identical."""
    P = ics.galaxy(seed=2)
    T = gpu_ctx.build(P)
    a1 = gpu_ctx.accel_grouped(T, None, theta=0.7, out_order=g.GT_OUT_ORIGINAL)
    a2 = gpu_ctx.accel_grouped(T, None, theta=0.7, G=2.0, out_order=g.GT_OUT_ORIGINAL)
    for u, v in zip(a1, a2):
        assert np.array_equal(2.0 * u, v)
    perm = np.random.default_rng(0).permutation(len(P["m"]))
    Pp = {k: v[perm] for k, v in P.items()}
    Tp = gpu_ctx.build(Pp)
    ap = gpu_ctx.accel_grouped(Tp, None, theta=0.7, out_order=g.GT_OUT_ORIGINAL)
    # particles with equal keys may swap, which only reorders FP32 sums inside a leaf: most forces
    # stay bit-identical, the rest move by summation-order rounding (amplified where the net force
    # nearly cancels)
    for u, v in zip(a1, ap):
        e = np.abs(u[perm] - v) / (np.abs(u[perm]) + 1e-300)
        assert np.median(e) == 0.0 and np.quantile(e, 0.999) <= 1e-6 and e.max() < 1e-3
    assert np.isfinite(a1[0]).all()


def test_host_outputs_copied_in_chunks_are_identical(gpu_ctx):
    """With host output arrays a large walk runs in chunks whose results are copied back while the
    next chunk runs; every group is walked exactly as in one launch, so the results are
    bit-identical to the device-output walk (all targets, explicit targets, with the potential)."""
    import torch

    P = ics.plummer(n=400000, seed=12, soft=0.01)
    T = gpu_ctx.build(P)
    nl = T.info()["n_live"]
    a_dev = gpu_ctx.accel_grouped(T, None, theta=0.6, want_phi=True, device_out=True, group_mode=g.GT_GROUP_BATCH,
                                  batch=32)
    a_host = gpu_ctx.accel_grouped(T, None, theta=0.6, want_phi=True, group_mode=g.GT_GROUP_BATCH, batch=32)
    for d, h in zip(a_dev, a_host):
        assert np.array_equal(d.cpu().numpy()[:nl], h)
    tg = np.sort(np.random.default_rng(3).choice(400000, 300000, replace=False)).astype(np.uint32)
    b_host = gpu_ctx.accel_grouped(T, tg, theta=0.6)
    b_dev = gpu_ctx.accel_grouped(T, torch.as_tensor(tg.view(np.int32), device="cuda"), theta=0.6)
    for d, h in zip(b_dev, b_host):
        assert np.array_equal(d.cpu().numpy(), h)


def test_host_aold_uploaded_in_chunks_is_identical(gpu_ctx):
    """A walk given a host aold and host outputs uploads aold piece by piece on the copy stream,
    each chunk waiting only for its own targets' piece, and downloads each chunk's results while the
    next one runs.  The results are bit-identical to the same walk with aold and the outputs on the
    device: grouped windows, the tidal tensor, and the per-target walk (explicit targets)."""
    import torch

    P = ics.plummer(n=400000, seed=15, soft=0.01)
    T = gpu_ctx.build(P)
    nl = T.info()["n_live"]
    kw = dict(group_mode=g.GT_GROUP_BATCH, batch=32)
    aold = gpu_ctx.form_aold(*gpu_ctx.accel_grouped(T, None, theta=0.7, **kw), 0.0025)
    aold_d = torch.as_tensor(aold, device="cuda")
    dev = tuple(torch.empty(nl, dtype=torch.float64, device="cuda") for _ in range(3))
    gpu_ctx.accel_grouped(T, None, aold=aold_d, outs=dev + (None,), **kw)
    host = gpu_ctx.accel_grouped(T, None, aold=aold, **kw)
    for d, h in zip(dev, host):
        assert np.array_equal(d.cpu().numpy(), h)

    tid = torch.empty((nl, 6), dtype=torch.float64, device="cuda")
    gpu_ctx.accel_grouped_ext(T, None, aold=aold_d, outs=dev + (None, tid, None), **kw)
    hx = gpu_ctx.accel_grouped_ext(T, None, aold=aold, **kw)
    for d, h in zip(dev + (tid,), hx[:3] + (hx[4],)):
        assert np.array_equal(d.cpu().numpy(), h)

    tg = np.arange(len(P["m"]), dtype=np.uint32)
    aold_t = gpu_ctx.form_aold(*gpu_ctx.accel(T, tg, theta=0.7), 0.0025)
    h1 = gpu_ctx.accel(T, tg, aold=aold_t)
    d1 = gpu_ctx.accel(T, torch.as_tensor(tg.view(np.int32), device="cuda"),
                       aold=torch.as_tensor(aold_t, device="cuda"))
    for d, h in zip(d1, h1):
        assert np.array_equal(d.cpu().numpy(), h)


def test_walks_and_searches_from_several_threads(gpu_ctx):
    """Four host threads, each with its own context, walk and search one fresh tree at the same
    time: the group list and the search nodes it builds on first use are made once, under the
    tree's lock, and every thread gets the single-thread results."""
    from concurrent.futures import ThreadPoolExecutor

    P = ics.plummer(n=300000, seed=14, soft=0.01)
    rng = np.random.default_rng(2)
    cen = [rng.normal(0.0, 0.5, 5000) for _ in range(3)]
    rad = np.full(5000, 0.05)
    ref_tree = gpu_ctx.build(P)
    ref_w = gpu_ctx.accel_grouped(ref_tree, None, theta=0.6, group_mode=g.GT_GROUP_BATCH, batch=32)
    ref_s = gpu_ctx.ngb_search(ref_tree, *cen, rad)
    T = gpu_ctx.build(P)

    def work(_):
        ctx = g.Context(0)
        w = ctx.accel_grouped(T, None, theta=0.6, group_mode=g.GT_GROUP_BATCH, batch=32)
        s = ctx.ngb_search(T, *cen, rad)
        ctx.close()
        return w, s

    with ThreadPoolExecutor(4) as ex:
        for w, s in ex.map(work, range(4)):
            for a, b in zip(w, ref_w):
                assert np.array_equal(a, b)
            assert np.array_equal(s[0], ref_s[0]) and np.array_equal(s[1], ref_s[1])


def test_small_target_lists_group_in_one_launch(gpu_ctx, plummer_trees):
    """Up to 8192 explicit targets form their groups in one block (the sparse active sets of deep
    time bins); longer lists take the multi-kernel path.  Across the threshold the groups and the
    forces are the same: the first 8192 targets walked alone (one launch) and as the head of 8193
    targets (the scan path) agree bit for bit, for windows of 32 and for leaf groups (all groups
    but the last, which the 8193rd target may extend)."""
    T, O = plummer_trees
    ob = O.order()[0]
    aold = 0.0025 * np.ones(len(ob))
    a = gpu_ctx.accel_grouped(T, ob[:8192], aold=aold[:8192], batch=32, group_mode=g.GT_GROUP_BATCH)
    b = gpu_ctx.accel_grouped(T, ob[:8193], aold=aold[:8193], batch=32, group_mode=g.GT_GROUP_BATCH)
    for u, v in zip(a, b):
        assert np.array_equal(u, v[:8192])
    leaf = O.order()[2][ob]
    head = int(np.nonzero(leaf[:8192] != leaf[8191])[0][-1]) + 1  # first target of the last group
    a = gpu_ctx.accel_grouped(T, ob[:8192], aold=aold[:8192], batch=0, count=True)
    ga = gpu_ctx.stats()["groups"]
    b = gpu_ctx.accel_grouped(T, ob[:8193], aold=aold[:8193], batch=0)
    for u, v in zip(a, b):
        assert np.array_equal(u[:head], v[:head])
    assert ga == 1 + int(np.count_nonzero(leaf[1:8192] != leaf[:8191]))


@pytest.mark.parametrize("nt", [None, 30001, 30000])
def test_window_pairs_match_single_windows(gpu_ctx, plummer_trees, nt):
    """Windows of 17-32 targets are walked two per warp by default (walk_pair_kernel): a node is
    tested only against the windows whose own walk reaches it, so each window makes its own
    walk's decisions.  The interaction counts therefore equal the one-window walk's exactly, and
    the forces agree to FP32 summation order (a node accepted instead of opened would move a
    force by ~1e-3).  All live targets, and explicit lists with an odd number of windows whose
    last one holds 17 or 16 targets; with the relative criterion, Barnes-Hut and the potential."""
    T, O = plummer_trees
    ob = O.order()[0]
    tg = None if nt is None else ob[:nt]
    kw = dict(group_mode=g.GT_GROUP_BATCH, batch=32)
    boot = gpu_ctx.accel_grouped(T, tg, theta=0.7, **kw)
    aold = gpu_ctx.form_aold(*boot, 0.0025)
    for crit in (dict(aold=aold, theta=0.0), dict(theta=0.6)):
        for pot in (False, True):
            runs = {}
            for pairs in (True, False):
                res = gpu_ctx.accel_grouped(T, tg, want_phi=pot, count=True, window_pairs=pairs, **crit, **kw)
                runs[pairs] = (np.stack(res), gpu_ctx.stats())
                plain = gpu_ctx.accel_grouped(T, tg, want_phi=pot, window_pairs=pairs, **crit, **kw)
                assert np.array_equal(np.stack(plain), runs[pairs][0])  # counting changes nothing
            (p, sp), (u, su) = runs[True], runs[False]
            for k in ("nodes_visited", "multipole", "pairs"):
                assert sp[k] == su[k], (k, sp[k], su[k])
            # per target: |a_pair - a_single| / |a_single| (the potential on its own), floored at a
            # thousandth of the median magnitude where the net force nearly cancels
            for d, r in ((p[:3] - u[:3], u[:3]), (p[3:] - u[3:], u[3:])):
                if len(r) == 0:
                    continue
                nd, nr = np.linalg.norm(d, axis=0), np.linalg.norm(r, axis=0)
                e = nd / np.maximum(nr, 1e-3 * np.median(nr))
                assert np.median(e) < 1e-6 and e.max() < 1e-4, (np.median(e), e.max())
