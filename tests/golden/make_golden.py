"""Generate tests/golden/golden.npz from the REFERENCE itself.

Runs the reference's own shmem tree and Peano-Hilbert functions, compiled from the reference
sources into oracle/_ref/libgizmo_ref.so (``make -C oracle ref``), on small seeded inputs and
stores their outputs.  The reference ships no golden force vectors (its shmem tests print error
percentiles without asserting), so these fixtures are what pins the oracle restatement and the GPU
path to the reference's numbers.  Regenerate with:

    make -C oracle ref && python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from oracle import Reference  # noqa: E402

from gizmo_shared_memory_b200 import ics  # noqa: E402


def gas_scenario(R):
    """A Plummer sphere of gas (type 0), stars (type 4) and sinks (type 5).  Gas softenings are
    the distance to the 32nd neighbour (the adaptive kernel's support) and zeta is of the size that
    makes its terms a percent-level correction; stars and sinks keep a small fixed softening.
    Every 97th particle is massless.  Returns the inputs and the reference's walks on them."""
    from scipy.spatial import cKDTree

    P = ics.plummer(n=4096, seed=42, soft=0.01)
    rng = np.random.default_rng(5)
    X = np.stack([P["x"], P["y"], P["z"]], 1)
    dk, _ = cKDTree(X).query(X, k=33)
    t = np.where(rng.uniform(size=4096) < 0.7, 0, 4).astype(np.uint8)
    t[rng.choice(4096, 120, replace=False)] = 5
    P["soft"] = np.where(t == 0, dk[:, -1], 0.01)
    P["m"][::97] = 0.0
    P["type"] = t
    P["zeta"] = np.where(t == 0, 0.1 * (1.0 / 4096) ** 2 * P["soft"] ** 2 * rng.normal(0, 1, 4096), 0.0)
    out = {k: P[k] for k in ("x", "y", "z", "m", "soft", "type", "zeta")}
    T = R.build_gas(P)
    ob = T.order()[0]
    out["orderbuf"] = ob
    out["nsink"] = T.nsink()
    a0 = T.accel_grouped_gas(ob, 0.7, 1.0, 0)
    aold = 0.005 * np.sqrt(a0[0] ** 2 + a0[1] ** 2 + a0[2] ** 2)
    out["aold"] = aold
    for name, theta, batch, ao, rs in (("bh", 0.7, 0, None, 0.0), ("bh_sink", 0.7, 0, None, 0.3),
                                       ("rel_sink", 0.0, 0, aold, 0.3), ("b8_sink", 0.7, 8, None, 0.3)):
        a = T.accel_grouped_gas(ob, theta, 1.0, batch, aold=ao, sink_radius=rs)
        for k, v in zip(("ax", "ay", "az"), a):
            out[f"{name}_{k}"] = v
    sub = ob[::7].copy()
    out["sub"] = sub
    for k, v in zip(("ax", "ay", "az"), T.accel(sub, 0.5)):
        out[f"acc_{k}"] = v
    for k, v in zip(("ax", "ay", "az"), T.accel_brute(sub)):
        out[f"brute_{k}"] = v
    return out


def ngb_scenario(R):
    """Neighbour search and the density solve (shmem/hydro.cc) on a Plummer sphere whose first 6000
    particles are gas (type 0) and the rest stars (type 4), every 53rd massless: the reference's
    gather / reverse / pair lists for seeded centres and radii, its per-node hmax, and its density
    solve from a cold start (with the neighbour cache), from a warm start, and with a condition-
    number history; plus a periodic box."""
    P = ics.plummer(n=8192, seed=21, soft=0.01)
    P["m"][::53] = 0.0
    n_gas = 6000
    P["type"] = np.where(np.arange(8192) < n_gas, 0, 4).astype(np.uint8)
    P["zeta"] = np.zeros(8192)
    out = {k: P[k] for k in ("x", "y", "z", "m", "type")}
    out["n_gas"] = np.array([n_gas])
    T = R.build_gas(P)
    ob = T.order()[0]
    tg = ob[ob < n_gas].copy()
    out["targets"] = tg
    d = T.density(tg, 32.0, 0.05, cache=True)
    for k in ("h", "rho", "nngb", "iters", "cache_start", "cache_flat"):
        out[f"cold_{k}"] = d[k]
    w = T.density(tg, 32.0, 0.05, h_start=1.1 * d["h"])
    for k in ("h", "rho", "nngb", "iters"):
        out[f"warm_{k}"] = w[k]
    rng = np.random.default_rng(77)
    cond = np.where(rng.uniform(size=8192) < 0.2, rng.uniform(100, 3000, 8192), 10.0)
    out["cond"] = cond
    c = T.density(tg, 32.0, 0.05, cond_prev=cond)
    for k in ("h", "rho", "nngb", "iters"):
        out[f"cond_{k}"] = c[k]
    h = np.zeros(8192)
    h[tg] = d["h"]
    out["h_part"] = h
    out["hmax"] = T.init_hmax(h[:n_gas], n_gas)
    cen = [rng.uniform(-1.5, 1.5, 400) for _ in range(3)]
    cen[0][:100], cen[1][:100], cen[2][:100] = P["x"][tg[:100]], P["y"][tg[:100]], P["z"][tg[:100]]
    rad = rng.uniform(0.02, 0.6, 400)
    rad[:100] = d["h"][:100]
    for k, v in zip("xyz", cen):
        out[f"c{k}"] = v
    out["radius"] = rad
    for mode, name in ((0, "gather"), (1, "reverse"), (2, "pairs")):
        st, f = T.ngb_search(*cen, rad, mode=mode, h=h, n_gas=n_gas)
        out[f"{name}_start"], out[f"{name}_found"] = st, f
    # periodic box of side 2: the sphere folded into it
    Q = ics.plummer(n=8192, seed=22, soft=0.01)
    for k in "xyz":
        Q[k] = np.mod(Q[k], 2.0)
    for k in "xyz":
        out[f"box_{k}"] = Q[k]
    out["box_m"] = Q["m"]
    TB = R.build(Q)
    obb = TB.order()[0]
    st, f = TB.ngb_search(*cen, 0.5 * rad, box=2.0)
    out["box_gather_start"], out["box_gather_found"] = st, f
    b = TB.density(obb[:3000], 32.0, 0.05, box=2.0)
    out["box_targets"] = obb[:3000].copy()
    for k in ("h", "rho", "nngb", "iters"):
        out[f"box_{k}"] = b[k]
    # a 2-D sheet (z = 0) and a 1-D line (y = z = 0), jittered lattices with a density gradient:
    # the dimension-aware kernels and solve, on the targets away from the edges
    for dim, name in ((2, "d2"), (1, "d1")):
        r2 = np.random.default_rng(30 + dim)
        if dim == 2:
            g1 = (np.arange(64) + 0.5) / 64
            x, y = (a.ravel() for a in np.meshgrid(g1, g1, indexing="ij"))
            x = x + r2.uniform(-0.2, 0.2, x.size) / 64
            y = y + r2.uniform(-0.2, 0.2, y.size) / 64
        else:
            x = (np.arange(4096) + 0.5) / 4096
            x = x + r2.uniform(-0.2, 0.2, x.size) / 4096
            y = np.zeros_like(x)
        x = x ** 1.3  # a density gradient along x
        n = x.size
        Q = {"x": x, "y": y, "z": np.zeros(n), "m": np.full(n, 1.0 / n), "soft": np.full(n, 0.01)}
        TD = R.build(Q)
        obd = TD.order()[0]
        inner = (Q["x"][obd] > 0.15) & (Q["x"][obd] < 0.85)
        if dim == 2:
            inner &= (Q["y"][obd] > 0.15) & (Q["y"][obd] < 0.85)
        obd = obd[inner].copy()
        for k in ("x", "y", "z", "m"):
            out[f"{name}_{k}"] = Q[k]
        dd = TD.density(obd, 12.0 if dim == 2 else 5.0, 0.05, n_dims=dim)
        out[f"{name}_targets"] = obd
        for k in ("h", "rho", "nngb", "iters"):
            out[f"{name}_{k}"] = dd[k]
    return out


def main():
    R = Reference()
    R.set_threads(1)
    out = {}
    rng = np.random.default_rng(2024)

    # ---- keys: exhaustive at 1..3 bits per axis, random at 20 and 42 bits (system/peano.cc) ----
    for bits in (1, 2, 3):
        g = np.arange(1 << bits, dtype=np.uint64)
        X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
        X, Y, Z = X.ravel(), Y.ravel(), Z.ravel()
        ph = [R.peano_key(a, b, c, bits) for a, b, c in zip(X, Y, Z)]
        mo = [R.morton_key(a, b, c, bits) for a, b, c in zip(X, Y, Z)]
        out[f"keys{bits}_xyz"] = np.stack([X, Y, Z], 1)
        out[f"keys{bits}_ph"] = np.array(ph, np.uint64)
        out[f"keys{bits}_morton"] = np.array(mo, np.uint64)
    for bits in (20, 42):
        xyz = rng.integers(0, 1 << bits, size=(2000, 3), dtype=np.uint64)
        ph, mo = [], []
        for a, b, c in xyz:
            p, m = R.peano_and_morton_key(a, b, c, bits)
            ph.append(p)
            mo.append(m)
        out[f"keys{bits}_xyz"] = xyz
        out[f"keys{bits}_ph_hi"] = np.array([p >> 64 for p in ph], np.uint64)
        out[f"keys{bits}_ph_lo"] = np.array([p & ((1 << 64) - 1) for p in ph], np.uint64)
        out[f"keys{bits}_morton_hi"] = np.array([p >> 64 for p in mo], np.uint64)
        out[f"keys{bits}_morton_lo"] = np.array([p & ((1 << 64) - 1) for p in mo], np.uint64)
    xyz20 = rng.integers(0, 1 << 20, size=(2000, 3), dtype=np.uint64)
    out["morton20_xyz"] = xyz20
    out["morton20"] = np.array([R.morton20(a, b, c) for a, b, c in xyz20], np.uint64)
    d = rng.uniform(1.0, 2.0, 2000)
    out["d2i_in"] = d
    out["d2i_out"] = np.array([R.double_to_int(v) for v in d], np.uint64)

    # ---- kernels (shmem/tree.h:59-80) ----------------------------------------------------------
    h = 0.01
    r = np.array([0.25, 0.5, 0.75, 0.999, 1.0, 2.0]) * h
    out["spline_r"] = r
    out["spline_h"] = np.full_like(r, h)
    out["spline_f"] = np.array([R.spline_force_over_r(a, h) for a in r])
    out["spline_p"] = np.array([R.spline_potential(a, h) for a in r])

    # ---- a Plummer sphere: tree and walks ------------------------------------------------------
    P = ics.plummer(n=4096, seed=42, soft=0.01)
    P["m"][::97] = 0.0  # a few massless particles: left out of the tree (tree.cc:355-359)
    for k in ("x", "y", "z", "m", "soft"):
        out[f"plummer_{k}"] = P[k]
    T = R.build(P)
    nd = T.nodes()
    ob, rank, leaf = T.order()
    out["plummer_orderbuf"] = ob
    out["plummer_rank"] = rank
    out["plummer_leaf_of"] = leaf
    for k in ("cx", "cy", "cz", "mass", "size", "delta", "soft", "gcx", "gcy", "gcz", "first",
              "next", "plo", "phi", "parent", "w_s", "w_len", "w_soft"):
        out[f"plummer_node_{k}"] = nd[k]
    tg = ob
    ax, ay, az = T.accel_grouped(tg, 0.7, 1.0, 0)
    out["plummer_bh_ax"], out["plummer_bh_ay"], out["plummer_bh_az"] = ax, ay, az
    aold = 0.005 * np.sqrt(ax * ax + ay * ay + az * az)
    out["plummer_aold"] = aold
    bx, by, bz = T.accel_grouped(tg, 0.0, 1.0, 0, aold=aold)
    out["plummer_rel_ax"], out["plummer_rel_ay"], out["plummer_rel_az"] = bx, by, bz
    cx, cy, cz = T.accel_grouped(tg, 0.7, 1.0, 8)
    out["plummer_b8_ax"], out["plummer_b8_ay"], out["plummer_b8_az"] = cx, cy, cz
    sub = tg[::7].copy()
    out["plummer_sub"] = sub
    px, py, pz = T.accel(sub, 0.5)
    out["plummer_acc_ax"], out["plummer_acc_ay"], out["plummer_acc_az"] = px, py, pz
    out["plummer_phi"] = T.potential(sub, 0.5)
    qx, qy, qz = T.accel_brute(sub)
    out["plummer_direct_ax"], out["plummer_direct_ay"], out["plummer_direct_az"] = qx, qy, qz

    # ---- tidal tensor and jerk (tree.cc:811-880) on the same sphere with seeded velocities -----
    vrng = np.random.default_rng(99)
    vel = [vrng.normal(0.0, 0.5, 4096) for _ in range(3)]
    for k, v in zip("xyz", vel):
        out[f"plummer_v{k}"] = v
    TV = R.build(P, vel=vel)
    vc, vmax = TV.vel_moments()
    for k, v in zip("xyz", vc):
        out[f"plummer_vcom_{k}"] = v
    out["plummer_vmax"] = vmax
    for name, theta, batch, ao in (("bh", 0.7, 0, None), ("b8", 0.7, 8, None), ("rel", 0.0, 0, aold)):
        _, _, _, tt, jj = TV.accel_grouped_ext(tg, theta, 1.0, batch, aold=ao, tidal=True, jerk=True)
        out[f"plummer_{name}_tidal"] = tt
        out[f"plummer_{name}_jerk"] = jj

    # ---- tree reuse: incremental moments, refresh and a walk on the reused tree (tree.cc:211-329)
    sys.path.insert(0, HERE)
    import reuse_scenario as RS

    TR = R.build(P, vel=vel)
    TR.reuse_begin()
    leaf_r = TR.order()[2]
    evs = RS.events(P, vel)
    for kind, parts, arr, tau in evs:
        TR.events(kind, leaf_r[parts], a=arr.get("a"), x=arr.get("x"), v=arr.get("v"), f=arr.get("f"), tau=tau)
    TR.refresh(RS.TAU)
    st = TR.node_state(RS.TAU)
    for k, v in st.items():
        out[f"reuse_{k}"] = v
    xr, yr, zr = RS.positions_after(P, vel, evs)
    TR.set_positions(xr, yr, zr)
    rx, ry, rz = TR.accel_grouped(tg, 0.0, 1.0, 0, aold=aold)
    out["reuse_ax"], out["reuse_ay"], out["reuse_az"] = rx, ry, rz

    # ---- gas, stars and sinks: the adaptive-softening zeta terms of gas-gas pairs (tree.cc:39-53)
    #      and sink-direct opening (tree.cc:691-698, 772-778) ------------------------------------
    G_ = gas_scenario(R)
    for k, v in G_.items():
        out[f"gas_{k}"] = v

    # ---- neighbour search and the density solve (shmem/hydro.cc:37-327) ------------------------
    for k, v in ngb_scenario(R).items():
        out[f"ngb_{k}"] = v

    # ---- collocated particles: the level-20 leaf (tree.cc:89) ----------------------------------
    Q = ics.plummer(n=600, seed=7, soft=0.02)
    Q["x"][:40] = Q["x"][0]
    Q["y"][:40] = Q["y"][0]
    Q["z"][:40] = Q["z"][0]
    for k in ("x", "y", "z", "m", "soft"):
        out[f"colloc_{k}"] = Q[k]
    TQ = R.build(Q)
    obq, _, _ = TQ.order()
    out["colloc_nnodes"] = np.array([TQ.nnodes])
    ex, ey, ez = TQ.accel_grouped(obq, 0.7, 1.0, 0)
    out["colloc_orderbuf"] = obq
    out["colloc_ax"], out["colloc_ay"], out["colloc_az"] = ex, ey, ez

    # ---- the reference's own test program (shmem/test_tree.cc), its printed accuracy table ------
    import re
    import subprocess

    exe = os.path.join(ROOT, "oracle", "_ref", "test_tree")
    txt = subprocess.run([exe, "20000"], capture_output=True, text=True, check=True,
                         env=dict(os.environ, OMP_NUM_THREADS="4")).stdout
    acc = txt.split("=== build")[0]
    rows = re.findall(r"^\s+([0-9.]+)\s+([0-9.e+-]+)\s+([0-9.e+-]+)\s+([0-9.e+-]+)\s*$", acc, re.M)
    out["test_tree_table"] = np.array([[float(v) for v in r] for r in rows])

    # ---- the reference's shmem/bench_treeforce.cc on a synthetic state: its printed checksums ----
    import tempfile

    Ps, vel = ics.plummer_state()
    with tempfile.TemporaryDirectory() as d:
        state = os.path.join(d, "state.bin")
        ics.write_state(state, Ps, vel)
        exe = os.path.join(ROOT, "oracle", "_ref", "bench_treeforce")
        txt = subprocess.run([exe, state, "1"], capture_output=True, text=True, check=True,
                             env=dict(os.environ, OMP_NUM_THREADS="4")).stdout
    sums = re.findall(r"sum_a=(\S+) sum_t=(\S+) sum_j=(\S+)", txt)
    out["treeforce_sums"] = np.array([[float(v) for v in r] for r in sums])

    path = os.path.join(HERE, "golden.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path}: {len(out)} arrays, {os.path.getsize(path) / 1024:.0f} KiB")


if __name__ == "__main__":
    main()
