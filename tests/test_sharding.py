"""Multi-rank target sharding, on CPU with the gloo backend (world size 2).

Each rank builds the tree from the full particle set and walks its slice of the targets through
sharding.walk_shard -- the same host function bench.py --split targets uses on the GPU -- with the
oracle walk as the walker.  The slices are all-gathered only to check that together they equal the
single-rank walk exactly, for the bootstrap walk and for the relative criterion with aold.
"""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from gizmo_shared_memory_b200 import ics
from gizmo_shared_memory_b200.sharding import gather_slices, shard_ranges, walk_shard


def test_shard_ranges_cover_and_align():
    for n in (0, 1, 31, 32, 33, 1000, 65536, 65537):
        for world in (1, 2, 3, 8):
            r = shard_ranges(n, world, 32)
            assert r[0][0] == 0 and r[-1][1] == n
            for (a, b), (c, d) in zip(r, r[1:]):
                assert b == c and a <= b
            for a, _ in r[1:]:
                assert a % 64 == 0 or a == n  # two windows: the walk's window pairs stay whole
            sizes = [b - a for a, b in r]
            assert max(sizes) - min(sizes) <= 64 + (n % 64)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, os.path.join(root, "oracle"))
    from oracle import Restatement

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        P = ics.plummer(n=12000, seed=5, soft=0.01)
        T = Restatement().build(P)           # every rank builds the same tree
        ob = T.order()[0]

        def windows(t):
            s = np.arange(0, len(t) + 1, 32, dtype=np.int64)
            return s if s[-1] == len(t) else np.append(s, len(t))

        def walker(theta):
            return lambda tg, ao: np.stack(T.walk_groups(tg, windows(tg), theta, aold=ao)[:3])

        ok = True
        _, _, boot = walk_shard(walker(0.7), ob, None, rank, world, 32)
        parts = [None] * world
        dist.all_gather_object(parts, boot)   # check only
        full = np.stack([gather_slices([p[k] for p in parts], len(ob), world, 32) for k in range(3)])
        aold = 0.005 * np.sqrt((full ** 2).sum(axis=0))
        _, _, rel = walk_shard(walker(0.0), ob, aold, rank, world, 32)
        parts2 = [None] * world
        dist.all_gather_object(parts2, rel)
        if rank == 0:
            ok &= bool(np.array_equal(full, walker(0.7)(ob, None)))
            full2 = np.stack([gather_slices([p[k] for p in parts2], len(ob), world, 32) for k in range(3)])
            ok &= bool(np.array_equal(full2, walker(0.0)(ob, aold)))
            q.put(ok)
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_rank_gloo_shards_equal_single_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        ok = q.get(timeout=240)
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert ok
    assert all(p.exitcode == 0 for p in procs)
