"""The ceiling of any learned acceptance rule over the monopole walk, measured.

A learned multipole-acceptance criterion replaces the relative criterion's estimate of a node's
error, M L^2 / r^4 (shmem/tree.h:134-135), by a prediction.  The best such a rule can do is to
know every (window, node) error exactly.  gt_mac_ceiling walks with exactly that rule: inside a
band of the plain ratio rho it sums the node's particles for every target of the window and
accepts the node only if the monopole's worst relative error over the window is at most eps.

This script measures, on sampled whole windows of one workload:
  * the plain walk at several alpha (mode 0: the production walk's own decisions), and
  * the exact-label walk at several eps (mode 1),
each with its node visits, interactions and force error against the FP64 direct sum.  The
production walk's device time over the whole workload at the same alphas fits the cost model
t = a * visits + b * interactions, which turns the exact-label walk's counts into the time a
walk with a free, perfect predictor would take.  At equal sampled p99 the ratio of the two times
is the ceiling of the learned criterion's speed-up.

    python -m gizmo_shared_memory_b200.mac_ceiling --workload clustered_16m --out ceiling.json
"""
from __future__ import annotations

import argparse
import json
import math
import sys
import time

import numpy as np


def relerr(a, b):
    d = np.sqrt(sum((x - y) ** 2 for x, y in zip(a, b)))
    n = np.sqrt(sum(y ** 2 for y in b))
    return d / np.where(n > 0, n, 1.0)


def make(workload):
    from gizmo_shared_memory_b200 import ics

    if workload == "clustered_16m":
        return ics.soneira_peebles(seed=3)
    if workload == "galaxy_4m":
        return ics.galaxy(seed=2)
    if workload == "clustered_1m":
        return ics.soneira_peebles(levels=10, seed=8)
    raise SystemExit(f"unknown workload {workload}")


def interp_at(p99s, ys, target):
    """log-log interpolation of y at p99 = target along a sweep sorted by p99 (None outside)."""
    order = np.argsort(p99s)
    p = np.log(np.asarray(p99s)[order])
    y = np.log(np.asarray(ys)[order])
    t = math.log(target)
    if t < p[0] or t > p[-1]:
        return None
    return float(math.exp(np.interp(t, p, y)))


def main(argv=None):
    import torch

    import gizmo_shared_memory_b200 as g

    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--workload", default="clustered_16m")
    ap.add_argument("--windows", type=int, default=1024, help="sampled whole windows of 32 targets")
    ap.add_argument("--alphas", default="0.001,0.0015,0.0025,0.0035,0.005,0.007,0.01,0.014")
    ap.add_argument("--eps", default="3e-5,1e-4,2e-4,4e-4,7e-4,1e-3,1.5e-3,2.5e-3,4e-3,7e-3")
    ap.add_argument("--band", default="0.001,1000", help="rho band of the exact labels")
    ap.add_argument("--cost-exp", default="0", help="exponents of the cost-aware threshold to sweep")
    ap.add_argument("--modes", default="", help="modes 2-5 (one ingredient of the exact rule each) to sweep "
                                                "over the alphas of the plain criterion")
    ap.add_argument("--alpha", type=float, default=0.0025, help="the headline plain criterion")
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--out", default=None)
    args = ap.parse_args(argv)
    alphas = [float(a) for a in args.alphas.split(",")]
    epss = [float(e) for e in args.eps.split(",")]
    cexps = [float(c) for c in args.cost_exp.split(",")]
    band = tuple(float(b) for b in args.band.split(","))

    P = make(args.workload)
    n = len(P["m"])
    ctx = g.Context(0, torch_stream=True)
    dev = {k: torch.as_tensor(v, device="cuda") for k, v in P.items()}
    T = ctx.build(dev)
    nl = T.info()["n_live"]
    ob = T.download(nodes=False)["orderbuf"]
    W = dict(group_mode=g.GT_GROUP_BATCH, batch=32)
    out = tuple(torch.empty(nl, dtype=torch.float64, device="cuda") for _ in range(3))
    ctx.accel_grouped(T, None, theta=0.7, outs=out + (None,), **W)
    amag_dev = torch.sqrt(out[0] ** 2 + out[1] ** 2 + out[2] ** 2)
    amag = amag_dev.cpu().numpy()

    rng = np.random.default_rng(31)
    wins = np.sort(rng.choice(nl // 32, size=min(args.windows, nl // 32), replace=False))
    pos = (wins[:, None] * 32 + np.arange(32)[None, :]).ravel()
    ns = len(pos)
    t0 = time.time()
    ref = ctx.direct(P, ob[pos], want_phi=False)[:3]
    print(f"{args.workload}: N={n}, {len(wins)} windows ({ns} targets); FP64 direct {time.time() - t0:.1f} s",
          file=sys.stderr)

    rows = []
    # plain criterion: sampled counts and error (mode 0), and the production walk's device time
    # over the whole workload at the same alpha
    aold = torch.empty_like(amag_dev)
    stream = torch.cuda.current_stream()
    for a in alphas:
        (cx, cy, cz), c = ctx.mac_ceiling(T, amag, a, wins, mode=0)
        e = relerr((cx, cy, cz), ref)
        aold.copy_(a * amag_dev)
        ctx.accel_grouped(T, None, aold=aold, outs=out + (None,), count=True, **W)
        st = ctx.stats()
        times = []
        for r in range(args.reps + 1):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            ctx.accel_grouped(T, None, aold=aold, outs=out + (None,), async_=True, **W)
            e1.record(stream)
            torch.cuda.synchronize()
            if r:
                times.append(e0.elapsed_time(e1))
        rows.append({"rule": "plain", "alpha": a, "p99": float(np.quantile(e, 0.99)), "median": float(np.median(e)),
                     "visits_per_window": float(c[:, 0].mean()),
                     "ipp": float((c[:, 1].sum() + c[:, 2].sum()) / ns),
                     "full_visits": st["nodes_visited"], "full_inter": st["multipole"] + st["pairs"],
                     "full_ms": float(np.median(times))})
        print(json.dumps(rows[-1]), file=sys.stderr)

    # cost model t = a V + b I over the plain runs (whole workload), non-negative coefficients:
    # across alpha the visits and the interactions move together, so the split between them is
    # poorly determined; the ratios below hold for either attribution
    from scipy.optimize import nnls

    A = np.array([[r["full_visits"], r["full_inter"]] for r in rows], float)
    y = np.array([r["full_ms"] for r in rows])
    coef, _ = nnls(A, y)
    fit = A @ coef
    model = {"ms_per_visit": float(coef[0]), "ms_per_interaction": float(coef[1]),
             "max_rel_residual": float(np.max(np.abs(fit - y) / y))}
    print(json.dumps(model), file=sys.stderr)
    scale = nl / ns  # sampled windows -> whole workload
    groups = nl / 32

    for cexp, eps in [(c, e) for c in cexps for e in epss]:
        t0 = time.time()
        (cx, cy, cz), c = ctx.mac_ceiling(T, amag, args.alpha, wins, mode=1, eps=eps, band=band, cost_exp=cexp)
        e = relerr((cx, cy, cz), ref)
        V = c[:, 0].mean() * groups
        inter = (c[:, 1].sum() + c[:, 2].sum()) * scale
        rows.append({"rule": "exact", "cost_exp": cexp, "eps": eps, "p99": float(np.quantile(e, 0.99)),
                     "median": float(np.median(e)),
                     "visits_per_window": float(c[:, 0].mean()), "ipp": float((c[:, 1].sum() + c[:, 2].sum()) / ns),
                     "labelled_per_window": float(c[:, 3].mean()), "label_particles_per_window": float(c[:, 4].mean()),
                     "model_ms": float(coef[0] * V + coef[1] * inter), "walk_s": time.time() - t0})
        print(json.dumps(rows[-1]), file=sys.stderr)
    for mode, a in [(int(m), a) for m in filter(None, args.modes.split(",")) for a in alphas]:
        (cx, cy, cz), c = ctx.mac_ceiling(T, amag, a, wins, mode=mode)
        e = relerr((cx, cy, cz), ref)
        V = c[:, 0].mean() * groups
        inter = (c[:, 1].sum() + c[:, 2].sum()) * scale
        rows.append({"rule": f"mode{mode}", "alpha": a, "p99": float(np.quantile(e, 0.99)),
                     "median": float(np.median(e)), "visits_per_window": float(c[:, 0].mean()),
                     "ipp": float((c[:, 1].sum() + c[:, 2].sum()) / ns),
                     "model_ms": float(coef[0] * V + coef[1] * inter)})
        print(json.dumps(rows[-1]), file=sys.stderr)
    for r in rows:
        if r["rule"] == "plain":
            r["model_ms"] = float(coef[0] * r["visits_per_window"] * groups + coef[1] * r["ipp"] * nl)

    plain = [r for r in rows if r["rule"] == "plain"]
    head = min(plain, key=lambda r: abs(r["alpha"] - args.alpha))
    targets = sorted({head["p99"], 5e-3})
    compare = []
    families = [("exact", c) for c in cexps] + [(f"mode{m}", None) for m in filter(None, args.modes.split(","))]
    for (rule, cexp), tp in [(f, t) for f in families for t in targets]:
        exact = [r for r in rows if r["rule"] == rule and (cexp is None or r["cost_exp"] == cexp)]
        t_plain = interp_at([r["p99"] for r in plain], [r["full_ms"] for r in plain], tp)
        m_plain = interp_at([r["p99"] for r in plain], [r["model_ms"] for r in plain], tp)
        m_exact = interp_at([r["p99"] for r in exact], [r["model_ms"] for r in exact], tp)
        i_plain = interp_at([r["p99"] for r in plain], [r["ipp"] for r in plain], tp)
        i_exact = interp_at([r["p99"] for r in exact], [r["ipp"] for r in exact], tp)
        v_plain = interp_at([r["p99"] for r in plain], [r["visits_per_window"] for r in plain], tp)
        v_exact = interp_at([r["p99"] for r in exact], [r["visits_per_window"] for r in exact], tp)
        compare.append({"rule": rule, "cost_exp": cexp, "p99": tp, "plain_ms_measured": t_plain, "plain_ms_model": m_plain,
                        "exact_ms_model": m_exact, "plain_ipp": i_plain, "exact_ipp": i_exact,
                        "plain_visits_per_window": v_plain, "exact_visits_per_window": v_exact,
                        "ceiling_speedup": (m_plain / m_exact) if (m_plain and m_exact) else None,
                        "interaction_ratio": (i_plain / i_exact) if (i_plain and i_exact) else None,
                        "visit_ratio": (v_plain / v_exact) if (v_plain and v_exact) else None})
        print(json.dumps(compare[-1]), file=sys.stderr)
    res = {"workload": args.workload, "n": n, "windows": int(len(wins)), "targets": int(ns), "band": band,
           "cost_model": model, "rows": rows, "at_equal_p99": compare}
    print(json.dumps(res))
    if args.out:
        with open(args.out, "w") as f:
            json.dump(res, f, indent=1)
    ctx.close()


if __name__ == "__main__":
    main()
