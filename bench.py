#!/usr/bin/env python
"""Tree-force throughput on B200: particles/s of the all-active grouped walk.

Workload (default ``clustered_16m``): 16,777,216 equal-mass particles of a seeded Soneira-Peebles
hierarchy in the unit cube (eta=4, lambda=1.9, 12 levels, 10% uniform background, softening 1e-4).
Protocol (shmem/bench_treeforce.cc:35-58 and shmem/mfm.cc:743-751): build the tree, a first walk
with Barnes-Hut theta=0.7 and aold=0, aold = alpha*|a|/G, then the timed walks with the relative
criterion alone (alpha=0.0025).  One step = one walk over every particle (targets = orderbuf) with
inputs resident in HBM; ``value`` = particles walked / device time.  ``e2e`` repeats the step
through the C ABI with host buffers: each step copies positions, masses, softenings and aold from
pinned host memory, rebuilds the tree, walks, and copies the accelerations back.  Force error is
measured against an FP64 direct sum on a seeded 4096-particle sample.

--impl reference times the reference's own CPU walk (shmem::accel_grouped, batch 0, compiled from
the reference sources into oracle/_ref) on a bounded sample of whole leaf groups of the same
workload, with every host thread.

Other workloads: --workload plummer_batch_256 (256 systems in one forest, autotuned, one captured
graph), --workload extras_galaxy_4m (the tidal tensor, the jerk, the gas rules and tree reuse on the
4M galaxy), --workload density_galaxy_4m / density_clustered_16m (the density solve).

Multi-GPU (--gpus N under torchrun): by default (--split targets) the ranks share one system:
every rank builds the same tree and walks its slice of the tree order, aligned to window pairs
(gizmo_shared_memory_b200/sharding.py), and ``value`` is the system's particles over the max-over-ranks
step time ("scaling": "strong").  --split systems walks one independent system per rank (seed +
rank, "scaling": "weak").  There is no data-path collective in either: only the barrier and the max
over ranks of the timed region.

--workload activeset_galaxy_4m / activeset_clustered_16m: sparse active sets (one call's latency
at 0.01-10 % actives, scattered and compact, leaf groups and windows), next to the reference's
CPU walk on the same targets.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "tree-force particles/s at fixed p99 force error: learned-MAC vs plain walk"
FLOPS_PER_INTERACTION = 20  # r^2 5, rsqrt 1, r^-3 and m 3, h test 2, acceleration 6, potential 2, select 1
WORKLOADS = {
    "clustered_16m": dict(desc="Soneira-Peebles clustered box, N=16,777,216, eta=4, lambda=1.9, "
                               "12 levels, 10% uniform background, softening 1e-4", alpha=0.0025),
    "galaxy_4m": dict(desc="Hernquist halo 3,145,728 + exponential disk 1,048,576, softening "
                           "0.005/0.002", alpha=0.0025),
    "plummer_65k": dict(desc="Plummer sphere N=65,536, truncated at 20a, softening 0.01", alpha=0.005),
    "merger_67m": dict(desc="two isolated galaxies of 33,554,432 particles each (halo + disk, masses halved), "
                            "centres 20 scale radii apart, the second rotated at random", alpha=0.0025),
}


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def make_workload(name, seed_offset=0):
    from gizmo_shared_memory_b200 import ics

    if name == "clustered_16m":
        return ics.soneira_peebles(seed=3 + seed_offset)
    if name == "galaxy_4m":
        return ics.galaxy(seed=2 + seed_offset)
    if name == "plummer_65k":
        return ics.plummer(n=65536, seed=42 + seed_offset)
    if name == "merger_67m":
        return ics.merger(seed=5 + seed_offset)
    raise SystemExit(f"unknown workload {name}")


# ---------------------------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        # the raw samples; the JSON line carries their summary
        import tempfile

        out_dir = os.environ.get("GT_CLOCKS_DIR", tempfile.gettempdir())
        self.path = os.path.join(out_dir, f"clocks_rank{device_index}.csv")

    def start(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.fh,
                stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(smax)),
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------------------------
# CPU reference walk on a bounded sample
# ---------------------------------------------------------------------------------------------
def window_sample(orderbuf, batch, want, rng):
    """Whole windows of `batch` consecutive targets of orderbuf (the windows accel_grouped forms
    over targets = orderbuf, shmem/tree.cc:668-670), picked at random until the sample holds at
    least `want` targets; returned in tree order, so the reference's windows over the sample are
    the same windows."""
    nw = len(orderbuf) // batch
    k = int(min(nw, max(1, -(-want // batch))))
    w = np.sort(rng.choice(nw, size=k, replace=False))
    pos = (w[:, None] * batch + np.arange(batch)[None, :]).ravel()
    return orderbuf[pos].astype(np.uint32)


def leaf_group_sample(orderbuf, leaf_of, want, rng):
    """Whole leaf groups (consecutive orderbuf runs with one leaf), picked at random until the
    sample holds at least `want` targets; returned in tree order."""
    L = leaf_of[orderbuf]
    starts = np.concatenate([[0], np.nonzero(np.diff(L))[0] + 1])
    ends = np.concatenate([starts[1:], [len(L)]])
    pick = rng.permutation(len(starts))
    sizes = (ends - starts)[pick]
    k = int(np.searchsorted(np.cumsum(sizes), want)) + 1
    sel = np.sort(pick[:k])
    return np.concatenate([orderbuf[s:e] for s, e in zip(starts[sel], ends[sel])]).astype(np.uint32)


def reference_omp_env():
    """The reference's recommended OpenMP placement (shmem/README.md:47-51), set before its library,
    and with it its OpenMP runtime, is loaded."""
    os.environ.setdefault("OMP_PROC_BIND", "spread")
    os.environ.setdefault("OMP_PLACES", "cores")


class CpuReference:
    """oracle/_ref (the reference's own shmem tree) when built, else the oracle restatement."""

    def __init__(self):
        reference_omp_env()
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        from oracle import Reference, Restatement, reference_available

        self.kind = "reference" if reference_available() else "port"
        self.lib = Reference() if self.kind == "reference" else Restatement()
        self.cores = os.cpu_count() or 1
        if self.kind == "reference":
            self.lib.set_threads(self.cores)
        else:
            os.environ.setdefault("OMP_NUM_THREADS", str(self.cores))

    def build(self, P):
        t0 = time.perf_counter()
        T = self.lib.build(P)
        return T, time.perf_counter() - t0

    def walk(self, T, targets, aold, theta=0.0, batch=0):
        if self.kind == "reference":
            return T.accel_grouped(targets, theta, 1.0, batch, aold=aold)
        return T.accel_grouped(targets, theta, 1.0, batch, aold=aold)[:3]

    def direct(self, T, P, targets):
        """FP64 direct sum: the reference's own accel_brute (shmem/tree.cc:946-971)."""
        if self.kind == "reference":
            return T.accel_brute(targets, 1.0)
        return self.lib.direct(P, targets)[:3]


def ph_order(P):
    """Live particles in Peano-Hilbert order of shmem::build's 20-bit cells, ties in index order:
    the GPU tree's order.  The keys come from the oracle's key function, which is pinned bit-exact
    to the reference's peano_hilbert_key (system/peano.cc:297-313)."""
    from oracle import Restatement

    keys, _ = Restatement().keys20(P, key_mode=1)
    live = np.nonzero(np.asarray(P["m"]) > 0)[0]
    return live[np.argsort(keys[live], kind="stable")].astype(np.uint32)


def sample_groups(T, batch, want, rng, order=None):
    ob, _, leaf = T.order()
    if batch > 0:
        return window_sample(ob if order is None else order, batch, want, rng)
    return leaf_group_sample(ob, leaf, want, rng)


def cpu_sample_walk(cpu, T, aold_orig, seconds, rng, alpha=None, batch=0, order=None):
    """Time one walk over a sample of whole groups (windows of `batch` consecutive targets of
    `order` -- the reference's own tree order by default -- or leaf groups for batch 0) sized to
    about `seconds` of CPU work."""
    tg = sample_groups(T, batch, 4096, rng, order)

    def aold_for(t):
        if aold_orig is not None:
            return aold_orig[t]
        a = cpu.walk(T, t, None, theta=0.7, batch=batch)
        return alpha * np.sqrt(a[0] ** 2 + a[1] ** 2 + a[2] ** 2)

    t0 = time.perf_counter()
    cpu.walk(T, tg, aold_for(tg), batch=batch)
    dt = time.perf_counter() - t0
    want = int(min(T.nlive, max(4096, len(tg) * seconds / max(dt, 1e-4))))
    tg = sample_groups(T, batch, want, rng, order)
    return tg, aold_for(tg)


def error_sample(n, rank=0):
    """The seeded 4096-particle sample both arms score against the FP64 direct sum."""
    rng = np.random.default_rng(77 + rank)
    return np.sort(rng.choice(n, size=min(4096, n), replace=False)).astype(np.uint32)


def reference_error(cpu, T, P, alpha, batch, order=None):
    """The reference walk's force error on the seeded sample: the groups holding the sampled
    particles (whole windows of `order`, or whole leaf groups) are walked as in the timed steps --
    bootstrap theta = 0.7, aold = alpha |a|, then the relative criterion -- and scored against the
    reference's own FP64 direct sum (the recipe of shmem/mfm.cc:2713-2789)."""
    n = len(P["m"])
    sample = error_sample(n)
    ob, rank, leaf = T.order()
    if order is not None:
        ob = order
        rank = np.zeros(n, np.int64)
        rank[ob] = np.arange(len(ob))
    if batch > 0:
        w = np.unique(rank[sample] // batch)
        pos = (w[:, None] * batch + np.arange(batch)[None, :]).ravel()
        pos = pos[pos < len(ob)]
    else:
        lv = leaf[ob]
        keep = np.isin(lv, np.unique(leaf[sample]))
        pos = np.nonzero(keep)[0]
    tg = ob[pos].astype(np.uint32)
    a = cpu.walk(T, tg, None, theta=0.7, batch=batch)
    aold = alpha * np.sqrt(a[0] ** 2 + a[1] ** 2 + a[2] ** 2)
    a = cpu.walk(T, tg, aold, batch=batch)
    at = np.full(n, -1, np.int64)
    at[tg] = np.arange(len(tg))
    k = at[sample]
    t0 = time.perf_counter()
    ref = cpu.direct(T, P, sample)
    td = time.perf_counter() - t0
    err = relerr([a[c][k] for c in range(3)], ref)
    return {"vs": "FP64 direct sum (the reference's accel_brute)", "sample": int(len(sample)),
            "median": float(np.median(err)), "p99": float(np.quantile(err, 0.99)),
            "walked_targets": int(len(tg)), "direct_s": td}


def grouping_of(args):
    """accel_grouped's batch for the --group choice, and its description."""
    order = "Morton" if args.key == "morton" else "Peano-Hilbert"
    if args.group == "batch":
        return args.group_max, (f"windows of {args.group_max} consecutive targets in {order} tree order "
                                f"(accel_grouped batch {args.group_max})")
    if args.group == "leaf":
        return 0, "leaf groups (accel_grouped batch 0)"
    return None, f"tree nodes of at most {args.group_max} particles"


def workload_config(args, n):
    """The `config` object, identical in both arms for the same arguments."""
    cfg = WORKLOADS[args.workload]
    alpha = args.alpha if args.alpha is not None else cfg["alpha"]
    return {"workload": args.workload, "description": cfg["desc"], "n": int(n),
            "criterion": f"plain relative criterion alpha={alpha} after a theta=0.7 bootstrap walk",
            "mac": "plain", "grouping": grouping_of(args)[1],
            "l2": (f"inputs larger than L2: {n * 32 / 2**20:.0f} MiB of particles per walk" if n * 32 > 126 * 2**20
                   else f"{n * 32 / 2**20:.0f} MiB of particles per walk: fits in L2"),
            "parallelism": (f"{args.gpus} GPUs: one system, targets split by tree-order slice"
                            if args.split == "targets" else f"{args.gpus} GPUs: one system per GPU")
            if args.gpus > 1 else "1 GPU"}


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    cfg = WORKLOADS[args.workload]
    alpha = args.alpha if args.alpha is not None else cfg["alpha"]
    batch, _ = grouping_of(args)
    if batch is None:
        print(json.dumps({"impl": "reference", "unavailable": "node groups are not a reference grouping"}))
        return
    P = make_workload(args.workload)
    n = len(P["m"])
    cpu = CpuReference()
    T, tbuild = cpu.build(P)
    # windows over the same order as the GPU arm's: Peano-Hilbert (the targets' order is the
    # caller's choice in accel_grouped), or the reference's own Morton orderbuf with --key morton
    order = ph_order(P) if (batch > 0 and args.key == "peano") else None
    rng = np.random.default_rng(123)
    tg, aold = cpu_sample_walk(cpu, T, None, args.sample_seconds, rng, alpha=alpha, batch=batch, order=order)
    for _ in range(args.warmup):
        cpu.walk(T, tg, aold, batch=batch)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        cpu.walk(T, tg, aold, batch=batch)
        times.append(time.perf_counter() - t0)
    t = float(np.mean(times))
    value = len(tg) / t
    error = reference_error(cpu, T, P, alpha, batch, order)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "particles/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded; see config.description)", "config": workload_config(args, n),
        "cpu_baseline": {"value": value, "unit": "particles/s", "cores": cpu.cores, "kind": cpu.kind,
                         "sample": f"{len(tg)} of {n} targets in whole groups picked at random, "
                                   f"walked per step; particles/s over "
                                   f"the sample stands for the whole job; tree prebuilt ({tbuild:.1f} s "
                                   f"build, not timed)"},
        "e2e": {"value": value, "unit": "particles/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "error": error,
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------------------------
def relerr(a, b):
    d = np.sqrt(sum((x - y) ** 2 for x, y in zip(a, b)))
    n = np.sqrt(sum(y ** 2 for y in b))
    return d / np.where(n > 0, n, 1.0)


def walk_kernel_name(args):
    """The kernel a single-system walk of this grouping runs: windows of 17-32 targets are walked
    two per warp (walk_pair_kernel), everything else by walk_kernel."""
    return "walk_pair_kernel" if args.group == "batch" and 16 < args.group_max <= 32 else "walk_kernel"


def read_profile_traffic(workload, kernel):
    """dram bytes per walk launch from the committed ncu summary, if one exists."""
    p = os.path.join(ROOT, "profiles", f"{kernel}_{workload}.json")
    try:
        return json.load(open(p)).get("dram_bytes_per_launch")
    except Exception:
        return None


def nominal_fp32(clocks, sms=148, lanes=128):
    """The FP32 CUDA-core peak from the data sheet arithmetic: SMs x FMA lanes x 2 flops x clock,
    at the maximum SM clock and at the median clock sampled during the timed steps."""
    mx = (clocks or {}).get("sm_max_mhz") or 1965.0
    med = (clocks or {}).get("sm_mhz") or mx
    return {"at_max_clock": sms * lanes * 2 * mx * 1e6 / 1e12, "at_sampled_clock": sms * lanes * 2 * med * 1e6 / 1e12,
            "sm_max_mhz": mx, "sm_mhz_sampled": med}


def window_parity(cpu, Tc, ob_gpu, aold_tree, full, batch, n_windows=256, seed=9):
    """This walk against the reference's accel_grouped on whole windows of this walk's own groups:
    the windows are passed in this tree's order with the same batch, so the reference forms exactly
    these windows (shmem/tree.cc:668-670), with the same aold.  `full` holds this walk's
    accelerations by particle index."""
    rng = np.random.default_rng(seed)
    nw = len(ob_gpu) // batch
    w = np.sort(rng.choice(nw, size=min(n_windows, nw), replace=False))
    pos = (w[:, None] * batch + np.arange(batch)[None, :]).ravel()
    tg = ob_gpu[pos].astype(np.uint32)
    r = cpu.walk(Tc, tg, aold_tree[pos], batch=batch)
    e = relerr([full[c][tg] for c in range(3)], r)
    return {"vs": f"the reference's accel_grouped ({cpu.kind}) on the same windows and aold",
            "targets": int(len(tg)), "median": float(np.median(e)), "p99": float(np.quantile(e, 0.99)),
            "max": float(e.max())}


def warm_build_ms(ctx, dev, offsets=None, reps=3, key_mode=0):
    """Device time of the tree build once the kernels are loaded and the memory pool holds the
    tree's arrays (the steady state of a rebuild every step); the first call also pays module
    loading and pool growth.  Median of `reps` rebuilds, per stage."""
    runs = []
    for _ in range(reps):
        T2 = ctx.build(dev, offsets=offsets, key_mode=key_mode)
        runs.append(T2.info()["build_ms"])
        T2.free()
    return {k: float(np.median([r[k] for r in runs])) for k in runs[0]}


MAC_MODEL = os.path.join(ROOT, "gizmo_shared_memory_b200", "mac_node_model.npy")


def learned_at_equal_p99(args, ctx, g, T, aold, wopts, sample, dref, p99_target, nl, world, dist):
    """The per-node learned criterion (GT_MAC_NODE, model trained on the Plummer and galaxy
    workloads by gizmo_shared_memory_b200/train_mac.py) at the largest kappa whose sampled p99 on
    the same 4096 targets does not exceed the plain walk's, timed like the plain walk."""
    import torch

    if not os.path.exists(MAC_MODEL):
        return {"unavailable": "no trained model (python -m gizmo_shared_memory_b200.train_mac)"}
    model = np.load(MAC_MODEL).astype(np.float32)
    meta_path = os.path.splitext(MAC_MODEL)[0] + ".json"
    c0 = json.load(open(meta_path))["median_prediction"] if os.path.exists(meta_path) else 0.0
    smp = torch.as_tensor(sample.astype(np.int64), device="cuda")
    ref = np.stack(dref[:3])

    def p99_at(kappa):
        full = ctx.accel_grouped(T, None, aold=aold, out_order=g.GT_OUT_ORIGINAL, mac=g.GT_MAC_NODE,
                                 mac_model=model, mac_kappa=kappa, **wopts)
        got = np.stack([f[smp].cpu().numpy() for f in full])
        e = np.linalg.norm(got - ref, axis=0) / np.linalg.norm(ref, axis=0)
        return float(np.quantile(e, 0.99)), float(np.median(e))

    # bisection on log kappa: the accepted bracket end is the fastest criterion meeting the target
    lo, hi = math.log10(0.05) + c0, math.log10(5.0) + c0
    best = None
    for _ in range(9):
        mid = 0.5 * (lo + hi)
        p99, med = p99_at(10 ** mid)
        if p99 <= p99_target:
            best = (10 ** mid, p99, med)
            lo = mid
        else:
            hi = mid
    if best is None:
        return {"unavailable": "no kappa in the bracket met the plain walk's p99"}
    kappa, p99, med = best
    lw = dict(mac=g.GT_MAC_NODE, mac_model=model, mac_kappa=kappa, **wopts)
    nl_ = nl
    out = tuple(torch.empty(nl_, dtype=torch.float64, device="cuda") for _ in range(3))
    ctx.accel_grouped(T, None, aold=aold, outs=out + (None,), count=True, **lw)
    st = ctx.stats()
    for _ in range(3):
        ctx.accel_grouped(T, None, aold=aold, outs=out + (None,), async_=True, **lw)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        ctx.accel_grouped(T, None, aold=aold, outs=out + (None,), async_=True, **lw)
    e1.record(stream)
    torch.cuda.synchronize()
    t = e0.elapsed_time(e1) / 1e3 / args.steps
    if dist:
        tt = torch.tensor([t], device="cuda", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t = float(tt[0])
    return {"criterion": "per-node learned correction (GT_MAC_NODE), node-only features, trained on the "
                         "Plummer 65k and galaxy 4M workloads", "kappa": kappa, "p99": p99, "median": med,
            "p99_target": p99_target, "value": nl_ * world / t, "ms_per_step": 1e3 * t,
            "interactions_per_particle": (st["multipole"] + st["pairs"]) / nl_}


def run_gpu_arm(args):
    import torch

    import gizmo_shared_memory_b200 as g

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    torch.cuda.set_device(local)
    cfg = WORKLOADS[args.workload]
    alpha = args.alpha if args.alpha is not None else cfg["alpha"]
    group_mode = {"leaf": g.GT_GROUP_LEAF, "node": g.GT_GROUP_NODE, "batch": g.GT_GROUP_BATCH}[args.group]
    wopts = dict(group_mode=group_mode, group_max=args.group_max,
                 batch=args.group_max if args.group == "batch" else 0)

    # --split targets (N > 1): one system, every rank builds the same tree and walks its
    # slice of the tree order, aligned to window pairs (sharding.walk_shard); --split systems: one
    # independent system per rank
    split = args.split == "targets" and (world > 1 or args.shard_check)
    P = make_workload(args.workload, seed_offset=0 if split else rank)
    n = len(P["m"])
    dev = {k: torch.as_tensor(v, device="cuda") for k, v in P.items()}
    ctx = g.Context(local, torch_stream=True)
    peak32, peak64 = ctx.measure_peaks()
    key_mode = g.GT_KEY_MORTON if args.key == "morton" else g.GT_KEY_PEANO
    T = ctx.build(dev, key_mode=key_mode)
    info = T.info()
    nl = info["n_live"]
    build_cold = info["build_ms"]
    info["build_ms"] = warm_build_ms(ctx, dev, key_mode=key_mode)
    out = tuple(torch.empty(nl, dtype=torch.float64, device="cuda") for _ in range(3))
    # bootstrap walk (theta = 0.7, aold = 0), then aold = alpha |a| / G
    ctx.accel_grouped(T, None, theta=0.7, outs=out + (None,), **wopts)
    aold = ctx.form_aold(*out, alpha)
    if split:
        from gizmo_shared_memory_b200.sharding import shard_ranges, walk_shard

        ob_dev = torch.as_tensor(T.download(nodes=False)["orderbuf"].view(np.int32), device="cuda")
        sa, sb = shard_ranges(nl, world, args.group_max)[rank]
        out_s = tuple(torch.empty(max(sb - sa, 1), dtype=torch.float64, device="cuda") for _ in range(3))

        def shard_walk(**kw):
            walk = lambda tg, ao: ctx.accel_grouped(T, tg, aold=ao, theta=0.0, outs=out_s + (None,), **wopts, **kw)
            return walk_shard(walk, ob_dev, aold, rank, world, args.group_max)

        # counted walk: interactions as the reference counts them (SHMEM_COUNT_WALK)
        shard_walk(count=True)
        st = ctx.stats()

        def step():
            shard_walk(async_=True)
    else:
        ctx.accel_grouped(T, None, aold=aold, theta=0.0, outs=out + (None,), count=True, **wopts)
        st = ctx.stats()

        def step():
            ctx.accel_grouped(T, None, aold=aold, theta=0.0, outs=out + (None,), async_=True, **wopts)
    inter_rank = st["multipole"] + st["pairs"]
    inter = inter_rank
    if dist:
        it = torch.tensor([inter_rank], device="cuda", dtype=torch.float64)
        dist.all_reduce(it)
        inter = float(it[0])

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    stream = torch.cuda.current_stream()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    l0 = ctx.launches()
    torch.cuda.synchronize()
    e_start = torch.cuda.Event(enable_timing=True)
    e_end = torch.cuda.Event(enable_timing=True)
    e_start.record(stream)
    for a, b in evs:
        a.record(stream)
        step()
        b.record(stream)
    e_end.record(stream)
    torch.cuda.synchronize()
    launches = ctx.launches() - l0
    clocks = sampler.stop()
    t_total = e_start.elapsed_time(e_end) / 1e3
    t_kernel = float(np.mean([a.elapsed_time(b) for a, b in evs])) / 1e3
    if dist:
        tt = torch.tensor([t_total, t_kernel], device="cuda", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_total, t_kernel = float(tt[0]), float(tt[1])
    t_step = t_total / args.steps
    jobs = 1 if split else world  # systems walked per step, all ranks together
    value = nl * jobs / t_step

    # accuracy: FP64 direct sum on a seeded 4096-particle sample
    sample = error_sample(n, rank)
    full = ctx.accel_grouped(T, None, aold=aold, theta=0.0, out_order=g.GT_OUT_ORIGINAL, **wopts)
    full = [f.cpu().numpy() for f in full]
    dref = ctx.direct(P, sample)
    err = relerr([full[k][sample] for k in range(3)], dref[:3])
    err_med, err_p99 = float(np.median(err)), float(np.quantile(err, 0.99))

    # the learned criterion at the same sampled p99 (the metric's comparison)
    learned = None
    if not args.no_learned and world == 1:
        learned = learned_at_equal_p99(args, ctx, g, T, aold, wopts, sample, dref, err_p99, nl, jobs, dist)

    # end to end through the C ABI with host buffers (pinned), build + walk every step
    e2e = None
    if not args.no_e2e:
        pin = {k: torch.from_numpy(v).pin_memory().numpy() for k, v in P.items()}
        aold_tree = aold.cpu()
        aold_h = torch.empty(nl, dtype=torch.float64).pin_memory()
        aold_h.copy_(aold_tree)
        aold_h = aold_h.numpy()
        ho = [torch.empty(nl, dtype=torch.float64).pin_memory().numpy() for _ in range(3)]
        hctx = g.Context(local)
        if split:
            # the target list sits in pinned memory like the other host arrays of the step
            ob_h = torch.from_numpy(T.download(nodes=False)["orderbuf"].view(np.int32)).pin_memory().numpy().view(np.uint32)
            sh = [o[sa:sb] for o in ho]
        ttimes = []
        for it in range(args.warmup + args.steps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            T2 = hctx.build(pin, key_mode=key_mode)
            if split:
                # this rank's slice, host arrays in and out
                walk_shard(lambda tg, ao: hctx.accel_grouped(T2, tg, aold=ao, theta=0.0, outs=tuple(sh) + (None,),
                                                             **wopts), ob_h, aold_h, rank, world, args.group_max)
            else:
                hctx.accel_grouped(T2, None, aold=aold_h, theta=0.0, outs=tuple(ho) + (None,), **wopts)
            t1 = time.perf_counter()
            T2.free()
            if it >= args.warmup:
                ttimes.append(t1 - t0)
        te = float(np.mean(ttimes))
        if dist:
            tt = torch.tensor([te], device="cuda", dtype=torch.float64)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            te = float(tt[0])
        nw = (sb - sa) if split else nl  # targets this rank walks
        e2e = {"value": nl * jobs / te, "unit": "particles/s", "ms_per_step": 1e3 * te,
               "ms_per_step_median": 1e3 * float(np.median(ttimes)), "ms_per_step_max": 1e3 * float(np.max(ttimes)),
               "h2d_bytes_per_step": int(5 * 8 * n + 8 * nw + (4 * nw if split else 0)),
               "d2h_bytes_per_step": int(3 * 8 * nw),
               "includes": "H2D of x,y,z,m,soft,aold from pinned memory + tree build + walk + D2H of ax,ay,az"}
        hctx.close()

    # CPU baseline (rank 0 only, N=1 only): the reference walk on a bounded sample, and the
    # parity of this walk with the reference's on whole windows of this walk's own groups
    cpu_line = None
    parity = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = CpuReference()
        Tc, tbuild = cpu.build(P)
        ob_gpu = T.download(nodes=False)["orderbuf"]
        aold_tree = aold.cpu().numpy()
        aold_orig = np.zeros(n)
        aold_orig[ob_gpu] = aold_tree
        batch, _ = grouping_of(args)
        batch = 0 if batch is None else batch
        tg, ao = cpu_sample_walk(cpu, Tc, aold_orig, args.sample_seconds, np.random.default_rng(123),
                                 batch=batch, order=ob_gpu if batch > 0 else None)
        t0 = time.perf_counter()
        cpu.walk(Tc, tg, ao, batch=batch)
        tc = time.perf_counter() - t0
        cpu_line = {"value": len(tg) / tc, "unit": "particles/s", "cores": cpu.cores, "kind": cpu.kind,
                    "sample": f"{len(tg)} targets in whole groups of this walk's grouping picked at "
                              f"random, the same aold; tree prebuilt ({tbuild:.1f} s CPU build, not timed)"}
        if args.group == "batch":
            parity = window_parity(cpu, Tc, ob_gpu, aold_tree, full, args.group_max, n_windows=256)

    achieved = FLOPS_PER_INTERACTION * inter_rank / t_kernel / 1e12  # this GPU's walk kernel
    if learned and "value" in learned:
        learned["speedup_vs_plain"] = learned["value"] / value
        # the specified fallback: the learned criterion replaces the plain one only where it meets
        # the p99 target and is faster; otherwise the plain criterion stays
        learned["selected"] = "learned" if learned["value"] > value else "plain (fallback)"
        learned["ceiling"] = ("any acceptance rule over the monopole walk: 1.29x fewer interactions at "
                              "equal p99 with exact per-(window, node) error labels, measured by "
                              "gizmo_shared_memory_b200/mac_ceiling.py (not run by this bench)")
    line = {
        "metric": METRIC, "value": value, "unit": "particles/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t_step,
        "higher_is_better": True, "scaling": "strong" if split else "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded; see config.description)",
        "config": workload_config(args, n),
        "precision": "FP64 positions and group-relative offsets, FP32 interactions; FP32 partial sums "
                     "per interaction-list flush, Kahan-compensated across flushes; FP64 potential and "
                     "final sums",
        "tree_bytes": int(info["n_nodes"]) * 64,
        "parity": parity,
        "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak32, "unit": "TFLOP/s",
                     "frac": achieved / peak32, "traffic": read_profile_traffic(args.workload, walk_kernel_name(args)),
                     "peak_source": "measured FP32 FMA-chain probe on this GPU (gt_measure_peaks), "
                                    "not in MEASURED_PEAKS.json",
                     "nominal_fp32_tflops": nominal_fp32(clocks),
                     "frac_of_nominal": achieved / nominal_fp32(clocks)["at_max_clock"],
                     "flops_per_interaction": FLOPS_PER_INTERACTION, "kernel": walk_kernel_name(args),
                     "kernel_ms": 1e3 * t_kernel, "fp64_peak_tflops": peak64},
        "cpu_baseline": cpu_line,
        "e2e": e2e,
        "gpu_launches": launches,
        "clocks": clocks,
        "error": {"vs": "FP64 direct sum", "sample": int(len(sample)), "median": err_med, "p99": err_p99},
        "interactions_per_particle": inter / (nl * jobs),
        "interactions_per_s": inter / t_step,
        "walk_stats": {k: st[k] for k in ("groups", "nodes_visited", "multipole", "pairs", "max_stack")},
        "build_ms": info["build_ms"],
        "build_ms_first_call": build_cold,
        "learned": learned,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def run_batch_arm(args):
    """256 independent Plummer systems of uneven N in one forest: one build, the launch
    configuration picked by the autotuner under a sampled p99 target, then the all-active walk of
    every system captured once as a CUDA graph and replayed.  Also times the same systems walked
    one launch per system, to show what batching buys."""
    import torch

    import gizmo_shared_memory_b200 as g
    from gizmo_shared_memory_b200 import ics

    torch.cuda.set_device(0)
    alpha = args.alpha if args.alpha is not None else 0.005
    P, off, meta = ics.plummer_batch(seed=4)
    S = len(off) - 1
    n = len(P["m"])
    dev = {k: torch.as_tensor(v, device="cuda") for k, v in P.items()}
    ctx = g.Context(0, torch_stream=True)
    peak32, _ = ctx.measure_peaks()
    F = ctx.build(dev, offsets=off)
    info = F.info()
    nl = info["n_live"]
    build_cold = info["build_ms"]
    info["build_ms"] = warm_build_ms(ctx, dev, offsets=off)
    out = tuple(torch.empty(nl, dtype=torch.float64, device="cuda") for _ in range(3))
    ctx.accel_grouped(F, None, theta=0.7, outs=out + (None,), group_mode=g.GT_GROUP_BATCH, batch=32)
    aold = ctx.form_aold(*out, alpha)
    # per-system FP64 direct-sum sample, 16 targets per system (4096 in all)
    rng = np.random.default_rng(77)
    sample, ref = [], [[], [], []]
    for s in range(S):
        loc = np.sort(rng.choice(int(off[s + 1] - off[s]), 16, replace=False)).astype(np.uint32)
        d = ctx.direct({k: v[off[s]:off[s + 1]] for k, v in P.items()}, loc, want_phi=False)
        sample.append(loc + np.uint32(off[s]))
        for k in range(3):
            ref[k].append(d[k])
    sample = np.concatenate(sample)
    ref = [np.concatenate(r) for r in ref]
    t0 = time.perf_counter()
    best, entries = ctx.autotune(F, aold, sample=sample, ref=ref, p99_max=5e-3, reps=3)
    t_tune = time.perf_counter() - t0
    kw = {k: v for k, v in best.items()}
    plan = ctx.plan(F, aold, out, **kw)
    ctx.accel_grouped(F, None, aold=aold, outs=out + (None,), count=True, **kw)
    st = ctx.stats()
    inter = st["multipole"] + st["pairs"]
    for _ in range(max(args.warmup, 3)):
        plan.launch()
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    sampler = ClockSampler(0)
    sampler.start()
    time.sleep(0.3)
    l0 = ctx.launches()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        plan.launch()
    e1.record(stream)
    torch.cuda.synchronize()
    launches = ctx.launches() - l0
    clocks = sampler.stop()
    t_step = e0.elapsed_time(e1) / 1e3 / args.steps
    full = ctx.accel_grouped(F, None, aold=aold, out_order=g.GT_OUT_ORIGINAL, **kw)
    got = np.stack([f.cpu().numpy()[sample] for f in full])
    err = relerr(list(got), ref)
    per_sys = err.reshape(S, 16)
    # one launch per system, same systems, same criterion and options
    trees, aolds, outs = [], [], []
    ob = F.download(nodes=False)["orderbuf"]
    live, _ = F.systems()
    aold_h = aold.cpu().numpy()
    for s in range(S):
        Ts = ctx.build({k: v[int(off[s]):int(off[s + 1])] for k, v in dev.items()})
        trees.append(Ts)
        # the forest's aold, restricted to system s, is already in this tree's order
        aolds.append(torch.as_tensor(aold_h[live[s]:live[s + 1]], device="cuda"))
        m = int(live[s + 1] - live[s])
        outs.append(tuple(torch.empty(m, dtype=torch.float64, device="cuda") for _ in range(3)))
    assert np.array_equal(ob[live[0]:live[1]] - off[0], trees[0].download(nodes=False)["orderbuf"])

    def separate():
        for s in range(S):
            ctx.accel_grouped(trees[s], None, aold=aolds[s], outs=outs[s] + (None,), async_=True, **kw)

    separate()
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        separate()
    e1.record(stream)
    torch.cuda.synchronize()
    t_sep = e0.elapsed_time(e1) / 1e3 / args.steps
    achieved = FLOPS_PER_INTERACTION * inter / t_step / 1e12
    line = {
        "metric": METRIC, "value": nl / t_step, "unit": "particles/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * t_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded Plummer spheres)",
        "config": {"workload": "plummer_batch_256", "n": n, "systems": S,
                   "n_per_system": [int(x) for x in meta["n"]],
                   "description": "256 Plummer spheres, N log-uniform in [1024, 262144] rescaled to ~2^24 "
                                  "in all, a log-uniform in [0.5, 2], softening 0.01 a",
                   "criterion": f"plain relative criterion alpha={alpha} after a theta=0.7 bootstrap walk",
                   "launch": "forest build (one pass for all systems), autotuned options, all-active walk "
                             "of every system captured as one CUDA graph (gt_plan) and replayed",
                   "autotuned": {k: v for k, v in best.items() if k != "mac_model"},
                   "l2": f"inputs larger than L2: {n * 32 / 2**20:.0f} MiB of particles"},
        "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak32, "unit": "TFLOP/s",
                     "frac": achieved / peak32, "traffic": None,
                     "kernel": ("walk_pair_kernel" if kw.get("group_mode") == g.GT_GROUP_BATCH and
                                16 < kw.get("batch", 0) <= 32 and kw.get("mac", g.GT_MAC_PLAIN) != g.GT_MAC_LEARNED
                                else "walk_kernel")},
        "gpu_launches": launches, "clocks": clocks,
        "error": {"vs": "FP64 direct sum per system, 16 targets each", "sample": int(len(sample)),
                  "median": float(np.median(err)), "p99": float(np.quantile(err, 0.99)),
                  "worst_system_p99": float(np.max(np.quantile(per_sys, 0.99, axis=1)))},
        "interactions_per_particle": inter / nl, "interactions_per_s": inter / t_step,
        "one_launch_per_system": {"ms_per_step": 1e3 * t_sep, "value": nl / t_sep,
                                  "speedup_of_batching": t_sep / t_step},
        "autotune": {"seconds": t_tune, "candidates": len(entries),
                     "entries": [{k: (round(v, 6) if isinstance(v, float) else v) for k, v in e.items()}
                                 for e in entries]},
        "build_ms": info["build_ms"],
        "build_ms_first_call": build_cold,
    }
    print(json.dumps(line), flush=True)
    plan.free()


def run_extras_arm(args):
    """The reference's options beyond the plain walk, on the 4M galaxy with seeded velocities
    (windows of 32, relative criterion alpha=0.0025 after a theta=0.7 bootstrap walk):
      * the tidal tensor, and the tidal tensor with the jerk (shmem/bench_treeforce.cc's variants);
      * the gas rules: 70 % gas with adaptive-softening zeta, 1 % sinks, sink-direct radius 0.02;
      * tree reuse: a kick and a speed bound for every particle, refresh_walk_nodes, the drifted
        positions and a walk on the reused tree, against a rebuild (with velocities) and a walk.
    Device time per step with inputs resident.  The CPU baseline is the reference's own walk,
    plain, with the tidal tensor, and with both, on a bounded sample of leaf groups."""
    import torch

    import gizmo_shared_memory_b200 as g

    torch.cuda.set_device(0)
    wl = "galaxy_4m"
    cfg = WORKLOADS[wl]
    alpha = args.alpha if args.alpha is not None else cfg["alpha"]
    P = make_workload(wl)
    n = len(P["m"])
    rng = np.random.default_rng(11)
    vel = [rng.normal(0.0, 0.3, n) for _ in range(3)]
    dev = {k: torch.as_tensor(v, device="cuda") for k, v in P.items()}
    vdev = [torch.as_tensor(v, device="cuda") for v in vel]
    ctx = g.Context(0, torch_stream=True)
    T = ctx.build(dev)
    ctx.tree_velocities(T, *vdev)
    nl = T.info()["n_live"]
    wopts = dict(group_mode=g.GT_GROUP_BATCH, group_max=32, batch=32)

    def mk(*shape):
        return torch.empty(*shape, dtype=torch.float64, device="cuda")

    a3 = (mk(nl), mk(nl), mk(nl))
    ctx.accel_grouped(T, None, theta=0.7, outs=a3 + (None,), **wopts)
    aold = ctx.form_aold(*a3, alpha)
    tid, jk = mk(nl, 6), mk(nl, 3)
    stream = torch.cuda.current_stream()

    def timed(step):
        for _ in range(max(args.warmup, 3)):
            step()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / args.steps

    # the gas tree: the same particles, types and zeta attached
    ty = np.where(rng.uniform(size=n) < 0.7, 0, 4).astype(np.uint8)
    ty[rng.choice(n, n // 100, replace=False)] = 5
    zeta = np.where(ty == 0, 0.1 * P["m"] ** 2 * P["soft"] ** 2 * rng.normal(0.0, 1.0, n), 0.0)
    Tg = ctx.build(dev)
    ctx.tree_gas(Tg, ty, zeta)
    # the reused tree: every live particle's leaf, its kick (m a dt) and speed bound
    Tr = ctx.build(dev)
    ctx.tree_velocities(Tr, *vdev)
    dl = Tr.download(nodes=False)
    ob = dl["orderbuf"]
    leaf_live = torch.as_tensor(dl["leaf_of"][ob].astype(np.int32), device="cuda")
    obd = torch.as_tensor(ob.astype(np.int64), device="cuda")
    dt = 1e-4
    dp = torch.stack([dev["m"][obd] * a3[k] * dt for k in range(3)], 1).contiguous()
    speed = torch.sqrt(sum(vdev[k][obd] ** 2 for k in range(3))).float().contiguous()
    clock = {"tau": 0.0}

    def reuse_step():
        clock["tau"] += dt
        tau = clock["tau"]
        ctx.tree_events(Tr, 0, leaf_live, a=dp, tau=tau)
        ctx.tree_events(Tr, 2, leaf_live, f=speed)
        ctx.tree_refresh(Tr, tau)
        ctx.tree_particles(Tr, x=dev["x"] + vdev[0] * tau, y=dev["y"] + vdev[1] * tau, z=dev["z"] + vdev[2] * tau)
        ctx.accel_grouped(Tr, None, aold=aold, outs=a3 + (None,), async_=True, **wopts)

    def rebuild_step():
        clock["tau"] += dt
        tau = clock["tau"]
        moved = dict(dev, x=dev["x"] + vdev[0] * tau, y=dev["y"] + vdev[1] * tau, z=dev["z"] + vdev[2] * tau)
        Tb = ctx.build(moved)
        ctx.tree_velocities(Tb, *vdev)
        ctx.accel_grouped(Tb, None, aold=aold, outs=a3 + (None,), async_=True, **wopts)
        torch.cuda.synchronize()
        Tb.free()

    sampler = ClockSampler(0)
    sampler.start()
    time.sleep(0.3)
    l0 = ctx.launches()
    ms = {
        "plain": timed(lambda: ctx.accel_grouped(T, None, aold=aold, outs=a3 + (None,), async_=True, **wopts)),
        "tidal": timed(lambda: ctx.accel_grouped_ext(T, None, aold=aold, outs=a3 + (None, tid, None), async_=True,
                                                     **wopts)),
        "tidal_jerk": timed(lambda: ctx.accel_grouped_ext(T, None, aold=aold, outs=a3 + (None, tid, jk), async_=True,
                                                          **wopts)),
        "gas_sinks": timed(lambda: ctx.accel_grouped(Tg, None, aold=aold, outs=a3 + (None,), async_=True,
                                                     sink_direct_radius=0.02, **wopts)),
        "reuse_step": timed(reuse_step),
        "rebuild_step": timed(rebuild_step),
    }
    launches = ctx.launches() - l0
    clocks = sampler.stop()
    rows = {k: {"ms_per_step": v, "particles_per_s": nl / (v / 1e3)} for k, v in ms.items()}
    # force error against the FP64 direct sum on the seeded 4096-particle sample: the plain walk,
    # and the gas-rules walk against the direct sum with the same zeta terms
    sample = error_sample(n)
    full = [f.cpu().numpy() for f in ctx.accel_grouped(T, None, aold=aold, out_order=g.GT_OUT_ORIGINAL, **wopts)]
    e = relerr([full[k][sample] for k in range(3)], ctx.direct(P, sample, want_phi=False)[:3])
    fg = [f.cpu().numpy() for f in ctx.accel_grouped(Tg, None, aold=aold, out_order=g.GT_OUT_ORIGINAL,
                                                     sink_direct_radius=0.02, **wopts)]
    eg = relerr([fg[k][sample] for k in range(3)], ctx.direct_gas(P, sample, type=ty, zeta=zeta))
    error = {"vs": "FP64 direct sum (with the zeta terms for the gas walk)", "sample": int(len(sample)),
             "plain": {"median": float(np.median(e)), "p99": float(np.quantile(e, 0.99))},
             "gas": {"median": float(np.median(eg)), "p99": float(np.quantile(eg, 0.99))}}
    cpu = None
    if not args.no_cpu:
        reference_omp_env()
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        from oracle import Reference, reference_available

        if reference_available():
            R = Reference()
            R.set_threads(os.cpu_count() or 1)
            TR = R.build(P, vel=vel)
            obr, _, leafr = TR.order()
            tg = leaf_group_sample(obr, leafr, 200000, np.random.default_rng(5))
            a0 = TR.accel_grouped(tg, 0.7, 1.0, 0)
            ao = alpha * np.sqrt(a0[0] ** 2 + a0[1] ** 2 + a0[2] ** 2)
            cpu = {"cores": os.cpu_count(), "kind": "reference", "unit": "particles/s",
                   "sample": f"{len(tg)} targets in whole leaf groups picked at random, leaf groups (batch 0), "
                             "the tree built with velocities (not timed)"}
            for name, kw in (("plain", None), ("tidal", dict(tidal=True, jerk=False)),
                             ("tidal_jerk", dict(tidal=True, jerk=True))):
                t0 = time.perf_counter()
                if kw is None:
                    TR.accel_grouped(tg, 0.0, 1.0, 0, aold=ao)
                else:
                    TR.accel_grouped_ext(tg, 0.0, 1.0, 0, aold=ao, **kw)
                cpu[name] = len(tg) / (time.perf_counter() - t0)
            for name in ("plain", "tidal", "tidal_jerk"):
                rows[name]["vs_cpu_reference"] = rows[name]["particles_per_s"] / cpu[name]
    line = {
        "metric": "tree-force particles/s with the tidal tensor and jerk, the gas rules and tree reuse",
        "value": rows["tidal_jerk"]["particles_per_s"], "unit": "particles/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms["tidal_jerk"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded galaxy, seeded velocities and gas fractions)",
        "config": {"workload": "extras_galaxy_4m", "n": n, "description": cfg["desc"],
                   "criterion": f"plain relative criterion alpha={alpha} after a theta=0.7 bootstrap walk",
                   "grouping": "windows of 32 consecutive targets in Peano-Hilbert tree order",
                   "gas": "70 % gas with zeta = 0.1 m^2 h^2 N(0,1), 1 % sinks, sink-direct radius 0.02",
                   "reuse": "kick and speed bound for every live particle, refresh, drifted positions, walk",
                   "l2": f"inputs larger than L2: {n * 32 / 2**20:.0f} MiB of particles"},
        "rows": rows, "cpu_baseline": cpu, "gpu_launches": launches, "clocks": clocks, "error": error,
    }
    print(json.dumps(line), flush=True)


def run_density_arm(args):
    """The density solve (shmem::density, hydro.cc:150-327) on the GPU tree: every particle a
    target, warm-started from the converged h of a first solve (what every step after the first
    does), DesNumNgb 32, tolerance 0.05.  value = targets / device time with everything resident;
    e2e = the same call with host arrays (targets and h_start in, h, rho, counts out).  The CPU
    baseline is the reference's own density on a bounded sample of the same targets."""
    import torch

    import gizmo_shared_memory_b200 as g

    torch.cuda.set_device(0)
    wl = args.workload[len("density_"):]
    P = make_workload(wl)
    n = len(P["m"])
    dev = {k: torch.as_tensor(v, device="cuda") for k, v in P.items()}
    ctx = g.Context(0, torch_stream=True)
    T = ctx.build(dev, key_mode=g.GT_KEY_MORTON)
    dl = T.download()
    ob = dl["orderbuf"]
    nl = len(ob)
    # first guess from each target's leaf: DesNumNgb at the leaf's density
    leaf = dl["leaf_of"][ob]
    cnt = (dl["phi"] - dl["plo"])[leaf]
    h0 = 0.8 * dl["size"][leaf] * np.cbrt(16.0 / np.maximum(cnt, 1))
    tg = torch.as_tensor(ob.view(np.int32), device="cuda")  # uint32 indices, passed as raw 32-bit words
    first = ctx.density(T, tg, h_start=torch.as_tensor(h0, device="cuda"))
    hconv = first["h"].clone()
    for _ in range(max(args.warmup, 3)):
        ctx.density(T, tg, h_start=hconv)
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    sampler = ClockSampler(0)
    sampler.start()
    time.sleep(0.3)
    l0 = ctx.launches()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ms = []
    for _ in range(args.steps):
        e0.record(stream)
        r = ctx.density(T, tg, h_start=hconv)
        e1.record(stream)
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
    launches = (ctx.launches() - l0) // args.steps
    clocks = sampler.stop()
    t_step = float(np.mean(ms)) / 1e3
    iters = r["iters"].float().mean().item()
    # end to end with host arrays
    hh = hconv.cpu().numpy()
    ctx.density(T, ob, h_start=hh)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        rh = ctx.density(T, ob, h_start=hh)
    t_e2e = (time.perf_counter() - t0) / args.steps
    cpu = None
    if not args.no_cpu:
        try:
            reference_omp_env()
            sys.path.insert(0, os.path.join(ROOT, "oracle"))
            from oracle import Reference, reference_available

            if reference_available():
                R = Reference()
                TR = R.build(P)
                k = min(200000, nl)
                step = max(1, nl // k)
                sel, hs = ob[::step][:k], hh[::step][:k]
                TR.density(sel[:1000], 32.0, 0.05, h_start=hs[:1000])
                c0 = time.perf_counter()
                TR.density(sel, 32.0, 0.05, h_start=hs)
                tc = time.perf_counter() - c0
                cpu = {"value": k / tc, "unit": "targets/s", "cores": os.cpu_count(), "kind": "reference",
                       "sample": f"{k} targets (every {step}th in tree order), warm start from the GPU's converged h, "
                                 "shmem::density with every host thread"}
        except Exception as e:  # the reference library is optional on the box
            log("cpu baseline skipped:", e)
    line = {
        "metric": "density-solve targets/s (warm start)", "value": nl / t_step, "unit": "targets/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "n": n, "description": WORKLOADS[wl]["desc"],
                   "des_ngb": 32, "ngb_tol": 0.05, "start": "warm: the converged h of a first solve",
                   "l2": f"inputs larger than L2: {n * 32 / 2**20:.0f} MiB of particles"},
        "iterations_mean": iters, "first_solve_iterations_mean": first["iters"].float().mean().item(),
        "kept_mean": float(rh["nngb"].mean()),
        "roofline": {"bound": "latency", "achieved": None, "peak": None, "unit": None, "frac": None, "traffic": None,
                     "kernel": "density_kernel",
                     "note": "one thread per target follows the tree: a dependent chain of node and particle loads"},
        "e2e": {"value": nl / t_e2e, "unit": "targets/s", "h2d_bytes_per_step": nl * 12,
                "d2h_bytes_per_step": nl * 24},
        "cpu_baseline": cpu, "gpu_launches": launches, "clocks": clocks,
    }
    print(json.dumps(line), flush=True)


def run_activeset_arm(args):
    """Sparse active sets: the engine's deep-timebin steps, where only a scattered fraction of the
    particles needs a force (shmem/bench_activeset.cc:1-16; compute_gravity hands the walk the
    active targets in tree order, shmem/mfm.cc:698-732).  For each active fraction, scattered
    (random particles) and compact (one run of the tree order), and for leaf groups (batch 0, the
    engine's grouping) and windows of 32, this times one call:
      * device: targets, aold and outputs resident on the device (CUDA events, median of steps);
      * host: the same call through the C ABI with host arrays (wall clock, copies included);
      * cpu: the reference's own accel_grouped on the same targets and aold (every host thread).
    Also the parity of the GPU walk with the reference's on the scattered 1 % subset."""
    import torch

    import gizmo_shared_memory_b200 as g

    torch.cuda.set_device(0)
    wl = args.workload.replace("activeset_", "")
    cfg = WORKLOADS[wl]
    alpha = args.alpha if args.alpha is not None else cfg["alpha"]
    P = make_workload(wl)
    n = len(P["m"])
    dev = {k: torch.as_tensor(v, device="cuda") for k, v in P.items()}
    ctx = g.Context(0, torch_stream=True)
    T = ctx.build(dev)
    nl = T.info()["n_live"]
    ob = T.download(nodes=False)["orderbuf"]
    out = tuple(torch.empty(nl, dtype=torch.float64, device="cuda") for _ in range(3))
    ctx.accel_grouped(T, None, theta=0.7, outs=out + (None,), group_mode=g.GT_GROUP_BATCH, batch=32)
    aold_tree = ctx.form_aold(*out, alpha).cpu().numpy()
    aold_p = np.zeros(n)
    aold_p[ob] = aold_tree
    cpu = None if args.no_cpu else CpuReference()
    Tc = cpu.build(P)[0] if cpu else None
    rng = np.random.default_rng(41)
    stream = torch.cuda.current_stream()
    rows = []
    parity = None
    error = None
    sampler = ClockSampler(0)
    sampler.start()
    l0 = ctx.launches()
    for frac in (1e-4, 1e-3, 1e-2, 1e-1):
        k = max(1, int(round(frac * nl)))
        for layout in ("scattered", "compact"):
            if layout == "scattered":
                pos = np.sort(rng.choice(nl, size=k, replace=False))
            else:
                s0 = int(rng.integers(0, nl - k + 1))
                pos = np.arange(s0, s0 + k)
            tg = ob[pos].astype(np.uint32)
            ao = aold_tree[pos]
            tg_d = torch.as_tensor(tg.view(np.int32), device="cuda")
            ao_d = torch.as_tensor(ao, device="cuda")
            o_d = tuple(torch.empty(k, dtype=torch.float64, device="cuda") for _ in range(3))
            for grouping, kw in (("leaf", dict(group_mode=g.GT_GROUP_LEAF, batch=0)),
                                 ("window32", dict(group_mode=g.GT_GROUP_BATCH, batch=32))):
                ctx.accel_grouped(T, tg_d, aold=ao_d, outs=o_d + (None,), count=True, **kw)
                st = ctx.stats()
                for _ in range(3):
                    ctx.accel_grouped(T, tg_d, aold=ao_d, outs=o_d + (None,), async_=True, **kw)
                torch.cuda.synchronize()
                dts = []
                for _ in range(max(args.steps, 5)):
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record(stream)
                    ctx.accel_grouped(T, tg_d, aold=ao_d, outs=o_d + (None,), async_=True, **kw)
                    e1.record(stream)
                    torch.cuda.synchronize()
                    dts.append(e0.elapsed_time(e1))
                hts = []
                for _ in range(max(args.steps, 5)):
                    t0 = time.perf_counter()
                    res = ctx.accel_grouped(T, tg, aold=ao, **kw)
                    hts.append(1e3 * (time.perf_counter() - t0))
                row = {"fraction": frac, "targets": k, "layout": layout, "grouping": grouping,
                       "groups": st["groups"], "device_ms": float(np.median(dts)),
                       "host_ms": float(np.median(hts)),
                       "interactions_per_target": (st["multipole"] + st["pairs"]) / k}
                if cpu:
                    b = 0 if grouping == "leaf" else 32
                    cts = []
                    for _ in range(3):
                        t0 = time.perf_counter()
                        r = cpu.walk(Tc, tg, ao, batch=b)
                        cts.append(1e3 * (time.perf_counter() - t0))
                    row["cpu_ms"] = float(min(cts))
                    row["cpu_cores"] = cpu.cores
                    if frac == 1e-2 and layout == "scattered":
                        e = relerr(res, r)
                        pr = {"targets": k, "median": float(np.median(e)), "p99": float(np.quantile(e, 0.99))}
                        parity = dict(parity or {}, **{grouping: pr})
                if frac == 1e-2 and layout == "scattered" and grouping == "leaf":
                    sub = np.arange(0, k, max(1, k // 4096))[:4096]
                    d = ctx.direct(P, tg[sub], want_phi=False)
                    e = relerr([res[c][sub] for c in range(3)], d[:3])
                    error = {"vs": "FP64 direct sum", "walk": "1 % scattered, leaf groups", "sample": int(len(sub)),
                             "median": float(np.median(e)), "p99": float(np.quantile(e, 0.99))}
                rows.append(row)
                log(json.dumps(row))
    launches = ctx.launches() - l0
    clocks = sampler.stop()
    head = [r for r in rows if r["fraction"] == 1e-3 and r["layout"] == "scattered" and r["grouping"] == "leaf"][0]
    line = {"metric": "active-set walk latency (one call)", "value": head["device_ms"], "unit": "ms",
            "n_gpus": 1, "steps": args.steps, "warmup": 3, "ms_per_step": head["device_ms"],
            "higher_is_better": False, "scaling": "none", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded; see config.description)",
            "config": {"workload": args.workload, "description": cfg["desc"], "n": n,
                       "criterion": f"plain relative criterion alpha={alpha}",
                       "headline": "0.1 % scattered actives, leaf groups"},
            "rows": rows, "parity": parity, "error": error, "gpu_launches": launches, "clocks": clocks,
            "e2e": {"value": head["host_ms"], "unit": "ms", "h2d_bytes_per_step": head["targets"] * 12,
                    "d2h_bytes_per_step": head["targets"] * 24}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS) + ["plummer_batch_256", "extras_galaxy_4m"] +
                    ["density_" + w for w in ("galaxy_4m", "clustered_16m")] +
                    ["activeset_" + w for w in ("galaxy_4m", "clustered_16m")], default="clustered_16m",
                    help="plummer_batch_256: the batched many-system case (forest + autotuner + graph); "
                         "density_*: the density solve on that workload")
    ap.add_argument("--alpha", type=float, default=None)
    ap.add_argument("--group", choices=["leaf", "node", "batch"], default="batch",
                    help="leaf: accel_grouped batch 0; batch: windows of --group-max consecutive "
                         "targets in tree order (accel_grouped batch > 0); node: tree nodes of at "
                         "most --group-max particles")
    ap.add_argument("--group-max", type=int, default=32)
    ap.add_argument("--split", choices=["targets", "systems"], default="targets",
                    help="N > 1: targets = one system, every rank walks a slice (aligned to window pairs) of its "
                         "tree order; systems = one independent system per rank")
    ap.add_argument("--shard-check", action="store_true",
                    help="run the --split targets path at N = 1 too (one slice holding every target), to "
                         "check it against the ordinary walk on one GPU")
    ap.add_argument("--key", choices=["peano", "morton"], default="peano",
                    help="sort key of the tree: the window order of --group batch")
    ap.add_argument("--sample-seconds", type=float, default=8.0)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned-criterion comparison")
    args = ap.parse_args()
    if args.warmup < 3:
        log("warm-up raised to 3 steps (timing rule)")
        args.warmup = 3
    if args.impl == "reference":
        run_reference_arm(args)
    elif args.workload == "plummer_batch_256":
        run_batch_arm(args)
    elif args.workload.startswith("activeset_"):
        run_activeset_arm(args)
    elif args.workload.startswith("density_"):
        run_density_arm(args)
    elif args.workload == "extras_galaxy_4m":
        run_extras_arm(args)
    else:
        run_gpu_arm(args)


if __name__ == "__main__":
    main()
