"""Forests: many independent systems of uneven N built in one pass (gt_build_systems) and walked in
one launch.  Each system must come out exactly as if it had been built and walked alone with
gt_build: the same keys, order and cells, and bit-identical accelerations (the walk visits the same
nodes in the same order, only the node numbering differs), for windowed, leaf and explicit-target
walks.  Systems include an empty one and one with massless particles.  The neighbour search and
the density solve on the forest must likewise reproduce each system's own tree."""
import numpy as np
import pytest

import gizmo_shared_memory_b200 as g
from gizmo_shared_memory_b200 import ics

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def batch():
    P, off, meta = ics.plummer_batch(n_systems=12, n_min=200, n_max=20000, n_total=60000, seed=7,
                                     spacing=50.0)
    # make system 3 empty and give system 5 some massless particles
    ns = np.diff(off)
    keep = np.ones(len(P["m"]), bool)
    keep[off[3]:off[4]] = False
    P = {k: v[keep] for k, v in P.items()}
    ns[3] = 0
    off = np.concatenate([[0], np.cumsum(ns)]).astype(np.int64)
    P["m"] = P["m"].copy()
    P["m"][off[5]:off[6]:7] = 0.0
    return P, off


def split(P, off, s):
    return {k: v[off[s]:off[s + 1]] for k, v in P.items()}


@pytest.fixture(scope="module")
def forest(gpu_ctx, batch):
    P, off = batch
    F = gpu_ctx.build(P, key_mode=g.GT_KEY_MORTON, offsets=off)
    trees = [gpu_ctx.build(split(P, off, s), key_mode=g.GT_KEY_MORTON) for s in range(len(off) - 1)]
    return F, trees


def test_forest_structure_matches_separate_builds(gpu_ctx, batch, forest):
    P, off = batch
    F, trees = forest
    S = len(off) - 1
    inf = F.info()
    assert inf["n_systems"] == S
    live, roots = F.systems()
    nl = [t.info()["n_live"] for t in trees]
    assert np.array_equal(np.diff(live), nl)
    assert inf["n_live"] == sum(nl)
    assert inf["n_nodes"] == sum(t.info()["n_nodes"] for t in trees)
    d = F.download(nodes=True)
    keys = F.keys()
    for s, t in enumerate(trees):
        ti = t.info()
        if ti["n_live"] > 0:
            assert np.allclose(roots[s, :3], ti["center"], rtol=0, atol=0)
            assert roots[s, 3] == ti["side"]
        ds = t.download(nodes=False)
        seg = d["orderbuf"][live[s]:live[s + 1]].astype(np.int64) - off[s]
        assert np.array_equal(seg, ds["orderbuf"].astype(np.int64))
        assert np.array_equal(keys[live[s]:live[s + 1]], t.keys())
        # root s covers exactly this system's live particles
        assert d["plo"][s] == live[s] and d["phi"][s] == live[s + 1]
        assert d["parent"][s] == -1


@pytest.mark.parametrize("mode,batch_size", [(g.GT_GROUP_BATCH, 32), (g.GT_GROUP_LEAF, 0),
                                             (g.GT_GROUP_BATCH, 64)])
def test_forest_walk_bit_identical(gpu_ctx, batch, forest, mode, batch_size):
    P, off = batch
    F, trees = forest
    live, _ = F.systems()
    # one window per warp: a single tree's windows of 32 are otherwise walked two at a time,
    # which matches the one-window walk to FP32 rounding only
    kw = dict(group_mode=mode, batch=batch_size, out_order=g.GT_OUT_ORIGINAL, window_pairs=False)
    fx, fy, fz = gpu_ctx.accel_grouped(F, None, theta=0.7, **kw)
    for s, t in enumerate(trees):
        if live[s + 1] == live[s]:
            continue
        sx, sy, sz = gpu_ctx.accel_grouped(t, None, theta=0.7, **kw)
        m = P["m"][off[s]:off[s + 1]] > 0
        for a, b in ((fx, sx), (fy, sy), (fz, sz)):
            assert np.array_equal(a[off[s]:off[s + 1]][m], b[m])


def test_forest_relative_criterion_and_targets(gpu_ctx, batch, forest):
    """Relative criterion with per-target aold, and an explicit target list that visits the
    systems out of order (leaf groups): identical to the separate walks."""
    P, off = batch
    F, trees = forest
    S = len(off) - 1
    rng = np.random.default_rng(3)
    fx, fy, fz = gpu_ctx.accel_grouped(F, None, theta=0.7, group_mode=g.GT_GROUP_BATCH, batch=32,
                                       out_order=g.GT_OUT_ORIGINAL)
    aold_all = gpu_ctx.form_aold(fx, fy, fz, 0.005)
    order = rng.permutation(S)
    tl, al, ref = [], [], []
    for s in order:
        idx = np.nonzero(P["m"][off[s]:off[s + 1]] > 0)[0]
        if len(idx) == 0:
            continue
        sub = np.sort(rng.choice(idx, size=max(1, len(idx) // 3), replace=False)).astype(np.uint32)
        a = aold_all[off[s] + sub]
        r = gpu_ctx.accel_grouped(trees[s], sub, aold=a, group_mode=g.GT_GROUP_LEAF)
        tl.append(sub + np.uint32(off[s]))
        al.append(a)
        ref.append(np.stack(r))
    got = gpu_ctx.accel_grouped(F, np.concatenate(tl), aold=np.concatenate(al), group_mode=g.GT_GROUP_LEAF)
    assert np.array_equal(np.stack(got), np.concatenate(ref, axis=1))


def test_forest_accuracy_vs_direct(gpu_ctx, batch, forest):
    P, off = batch
    F, _ = forest
    fx, fy, fz = gpu_ctx.accel_grouped(F, None, theta=0.7, group_mode=g.GT_GROUP_BATCH, batch=32,
                                       out_order=g.GT_OUT_ORIGINAL)
    aold = gpu_ctx.form_aold(fx, fy, fz, 0.005)
    m = P["m"] > 0
    aold = np.where(m, aold, 0.0)
    live_idx = np.nonzero(m)[0].astype(np.uint32)
    ax, ay, az = gpu_ctx.accel_grouped(F, live_idx, aold=aold[live_idx], group_mode=g.GT_GROUP_BATCH,
                                       batch=32)
    errs = []
    for s in range(len(off) - 1):
        sel = live_idx[(live_idx >= off[s]) & (live_idx < off[s + 1])]
        if len(sel) == 0:
            continue
        pos = np.searchsorted(live_idx, sel)
        sample = sel[:: max(1, len(sel) // 64)]
        ps = np.searchsorted(live_idx, sample)
        dx, dy, dz = gpu_ctx.direct(split(P, off, s), (sample - off[s]).astype(np.uint32), want_phi=False)[:3]
        d = np.sqrt((ax[ps] - dx) ** 2 + (ay[ps] - dy) ** 2 + (az[ps] - dz) ** 2)
        errs.append(d / np.sqrt(dx * dx + dy * dy + dz * dz))
        assert len(pos) == len(sel)
    e = np.concatenate(errs)
    assert np.median(e) < 5e-3 and np.quantile(e, 0.99) < 2e-2


def test_forest_bad_offsets(gpu_ctx, batch):
    P, off = batch
    bad = off.copy()
    bad[-1] -= 1
    with pytest.raises(g.GTError) as e:
        gpu_ctx.build(P, offsets=bad)
    assert e.value.status == 1
    bad = off.copy()
    bad[2], bad[3] = bad[3], bad[2]
    if bad[2] != bad[3]:
        with pytest.raises(g.GTError):
            gpu_ctx.build(P, offsets=bad)
    # the context stays usable
    T = gpu_ctx.build(split(P, off, 0))
    assert T.info()["n_live"] > 0


def test_forest_with_gas_rules_bit_identical(gpu_ctx, batch):
    """Gas data on a forest (types with sinks, zeta): the zeta terms and the sink rule act per
    system exactly as on each system's own tree -- the per-node sink counts climb to each
    system's root -- so the accelerations are bit-identical to the separate gas walks."""
    P, off = batch
    n = len(P["m"])
    rng = np.random.default_rng(12)
    ty = np.where(rng.uniform(size=n) < 0.7, 0, 4).astype(np.uint8)
    ty[rng.choice(n, n // 50, replace=False)] = 5
    soft = P["soft"] * rng.uniform(1.0, 20.0, n)
    zeta = np.where(ty == 0, 0.1 * P["m"] ** 2 * soft ** 2 * rng.normal(0.0, 1.0, n), 0.0)
    Q = dict(P, soft=soft)
    F = gpu_ctx.build(Q, key_mode=g.GT_KEY_MORTON, offsets=off)
    gpu_ctx.tree_gas(F, ty, zeta)
    kw = dict(group_mode=g.GT_GROUP_BATCH, batch=32, out_order=g.GT_OUT_ORIGINAL, sink_direct_radius=0.5)
    fx, fy, fz = gpu_ctx.accel_grouped(F, None, theta=0.7, **kw)
    acted = False
    for s in range(len(off) - 1):
        sl = slice(off[s], off[s + 1])
        if not (P["m"][sl] > 0).any():
            continue
        t = gpu_ctx.build({k: v[sl] for k, v in Q.items()}, key_mode=g.GT_KEY_MORTON)
        gpu_ctx.tree_gas(t, ty[sl], zeta[sl])
        sx, sy, sz = gpu_ctx.accel_grouped(t, None, theta=0.7, **kw)
        m = P["m"][sl] > 0
        for a, b in ((fx, sx), (fy, sy), (fz, sz)):
            assert np.array_equal(a[sl][m], b[m])
        plain = gpu_ctx.build({k: v[sl] for k, v in Q.items()}, key_mode=g.GT_KEY_MORTON)
        px, _, _ = gpu_ctx.accel_grouped(plain, None, theta=0.7, **kw)
        acted |= not np.array_equal(px[m], sx[m])
    assert acted  # the gas rules changed some forces


def local_targets(P, off, S, rng, massless=True):
    """Per system (visited in random order) a sorted random subset of its particle indices,
    massless ones included when asked: the forest's global list and each system's local list."""
    glob, loc = [], {}
    for s in rng.permutation(S):
        n = off[s + 1] - off[s]
        if n == 0:
            continue
        pool = np.arange(n) if massless else np.nonzero(P["m"][off[s]:off[s + 1]] > 0)[0]
        sub = np.sort(rng.choice(pool, size=max(1, len(pool) // 3), replace=False)).astype(np.uint32)
        glob.append(sub + np.uint32(off[s]))
        loc[s] = sub
    return np.concatenate(glob), loc


@pytest.mark.parametrize("mode", [g.GT_GROUP_LEAF, g.GT_GROUP_SINGLE])
def test_forest_massless_targets_walk_their_own_system(gpu_ctx, batch, forest, mode):
    """Massless particles sit after every live one in tree order, outside every system's live
    range: an explicit target list holding massless particles must still walk each one in its own
    system, bit-identical to the separate walks."""
    P, off = batch
    F, trees = forest
    S = len(off) - 1
    rng = np.random.default_rng(11)
    tl, loc = local_targets(P, off, S, rng)
    assert np.any(P["m"][tl] == 0)
    got = np.stack(gpu_ctx.accel_grouped(F, tl, theta=0.7, group_mode=mode))
    k = 0
    for s in loc:
        r = np.stack(gpu_ctx.accel_grouped(trees[s], loc[s], theta=0.7, group_mode=mode))
        assert np.array_equal(got[:, k:k + len(loc[s])], r), s
        k += len(loc[s])
    assert k == len(tl)


def test_forest_neighbour_search(gpu_ctx, batch, forest):
    """A centre with no system named searches every system in turn: its gather (reverse) list is
    the concatenation, in system order, of the separate trees' gather (reverse) lists, indices
    shifted by the offsets, and its pair list all the gathers followed by all the reverses.  With a
    system named, exactly that system's lists."""
    P, off = batch
    F, trees = forest
    S = len(off) - 1
    rng = np.random.default_rng(5)
    n = len(P["m"])
    # centres on particles of every system, plus points between the systems
    pick = rng.choice(n, 300, replace=False)
    cen = [np.concatenate([P[k][pick], rng.uniform(P[k].min(), P[k].max(), 100)]) for k in "xyz"]
    rad = rng.uniform(0.05, 2.0, len(cen[0]))
    nc = len(rad)
    h = rng.uniform(0.05, 1.0, n)
    gpu_ctx.tree_hmax(F, h, n)
    for s, t in enumerate(trees):
        gpu_ctx.tree_hmax(t, h[off[s]:off[s + 1]], off[s + 1] - off[s])

    def lists(T, mode, hh, ng, shift, **kw):
        st, f = gpu_ctx.ngb_search(T, *cen, rad, mode=mode, h=hh, n_gas=ng, **kw)
        f = f.astype(np.int64) + shift
        return [f[st[c]:st[c + 1]] for c in range(nc)]

    per = {m: [lists(t, m, h[off[s]:off[s + 1]], off[s + 1] - off[s], off[s]) for s, t in enumerate(trees)]
           for m in (g.GT_NGB_GATHER, g.GT_NGB_REVERSE)}
    want = {m: [np.concatenate([per[m][s][c] for s in range(S)]) for c in range(nc)] for m in per}
    want[g.GT_NGB_PAIRS] = [np.concatenate([want[g.GT_NGB_GATHER][c], want[g.GT_NGB_REVERSE][c]])
                            for c in range(nc)]
    sysid = rng.integers(0, S, nc).astype(np.int32)
    for mode in (g.GT_NGB_GATHER, g.GT_NGB_REVERSE, g.GT_NGB_PAIRS):
        got = lists(F, mode, h, n, 0)
        for c in range(nc):
            assert np.array_equal(got[c], want[mode][c]), (mode, c)
        got = lists(F, mode, h, n, 0, systems=sysid)
        for c in range(nc):
            s = sysid[c]
            w = {g.GT_NGB_GATHER: per[g.GT_NGB_GATHER][s][c], g.GT_NGB_REVERSE: per[g.GT_NGB_REVERSE][s][c]}
            w[g.GT_NGB_PAIRS] = np.concatenate([w[g.GT_NGB_GATHER], w[g.GT_NGB_REVERSE]])
            assert np.array_equal(got[c], w[mode]), (mode, c)
    assert sum(len(x) for x in want[g.GT_NGB_GATHER]) > 10 * nc
    with pytest.raises(g.GTError):
        gpu_ctx.ngb_search(F, *cen, rad, systems=np.full(nc, S, np.int32))

def test_forest_density(gpu_ctx, batch, forest):
    """Each density target searches the system that owns it, from that system's own default h
    (the mean density of its own particles): bit-identical to the separate solves, cold and warm,
    massless targets included."""
    P, off = batch
    F, trees = forest
    S = len(off) - 1
    rng = np.random.default_rng(9)
    tl, loc = local_targets(P, off, S, rng)
    d = gpu_ctx.density(F, tl, des_ngb=32.0)
    k = 0
    hs = np.empty(len(tl))
    for s in loc:
        r = gpu_ctx.density(trees[s], loc[s], des_ngb=32.0)
        seg = slice(k, k + len(loc[s]))
        for key in ("h", "rho", "nngb", "iters"):
            assert np.array_equal(d[key][seg], r[key]), (s, key)
        hs[seg] = 1.2 * r["h"]
        k += len(loc[s])
    w = gpu_ctx.density(F, tl, des_ngb=32.0, h_start=hs)
    k = 0
    for s in loc:
        seg = slice(k, k + len(loc[s]))
        r = gpu_ctx.density(trees[s], loc[s], des_ngb=32.0, h_start=hs[seg])
        for key in ("h", "rho", "nngb", "iters"):
            assert np.array_equal(w[key][seg], r[key]), (s, key)
        k += len(loc[s])


def test_forest_window_pairs_match_single_windows(gpu_ctx, batch, forest):
    """A forest's windows are walked two per warp like a single tree's; two windows of different
    systems start from their own roots.  Each window still tests exactly its own nodes: the
    counts equal the one-window walk's, the forces agree to FP32 summation order.  All live
    targets and an explicit list that visits the systems out of order."""
    P, off = batch
    F, _ = forest
    S = len(off) - 1
    kw = dict(group_mode=g.GT_GROUP_BATCH, batch=32)
    boot = gpu_ctx.accel_grouped(F, None, theta=0.7, window_pairs=False, out_order=g.GT_OUT_ORIGINAL, **kw)
    aold = gpu_ctx.form_aold(*boot, 0.0025)  # per particle index
    ob = F.download(nodes=False)["orderbuf"][:F.info()["n_live"]]
    tl, _ = local_targets(P, off, S, np.random.default_rng(21), massless=False)
    for tg in (None, tl):
        a = aold[ob] if tg is None else aold[tl]  # per target, in the order walked
        runs = {}
        for pairs in (True, False):
            res = gpu_ctx.accel_grouped(F, tg, aold=a, count=True, window_pairs=pairs, **kw)
            runs[pairs] = (np.stack(res), gpu_ctx.stats())
        (p, sp), (u, su) = runs[True], runs[False]
        for k in ("nodes_visited", "multipole", "pairs"):
            assert sp[k] == su[k], (k, sp[k], su[k])
        nd, nr = np.linalg.norm(p - u, axis=0), np.linalg.norm(u, axis=0)
        e = nd / np.maximum(nr, 1e-3 * np.median(nr))
        assert np.median(e) < 1e-6 and e.max() < 1e-4, (np.median(e), e.max())
