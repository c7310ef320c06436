"""Multi-rank target sharding, on CPU with the gloo backend (world size 2).

Each rank builds the tree from the full particle set, walks its slice of the targets with the
oracle walk (the GPU walk's host-side logic is the same: a contiguous tree-order slice on window
edges), and the slices are all-gathered only to check that together they equal the single-rank
walk exactly.
"""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from gizmo_shared_memory_b200 import ics
from gizmo_shared_memory_b200.sharding import gather_slices, rank_targets, shard_ranges


def test_shard_ranges_cover_and_align():
    for n in (0, 1, 31, 32, 33, 1000, 65536, 65537):
        for world in (1, 2, 3, 8):
            r = shard_ranges(n, world, 32)
            assert r[0][0] == 0 and r[-1][1] == n
            for (a, b), (c, d) in zip(r, r[1:]):
                assert b == c and a <= b
            for a, _ in r[1:]:
                assert a % 32 == 0 or a == n
            sizes = [b - a for a, b in r]
            assert max(sizes) - min(sizes) <= 32 + (n % 32)


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
        mine = rank_targets(ob, rank, world, 32)
        starts = np.arange(0, len(mine) + 1, 32, dtype=np.int64)
        if starts[-1] != len(mine):
            starts = np.append(starts, len(mine))
        ax, ay, az, _, _ = T.walk_groups(mine, starts, 0.7)
        parts = [None] * world
        dist.all_gather_object(parts, np.stack([ax, ay, az]))   # check only
        if rank == 0:
            full = np.stack([gather_slices([p[k] for p in parts], len(ob), world, 32) for k in range(3)])
            starts_all = np.arange(0, len(ob) + 1, 32, dtype=np.int64)
            if starts_all[-1] != len(ob):
                starts_all = np.append(starts_all, len(ob))
            bx, by, bz, _, _ = T.walk_groups(ob, starts_all, 0.7)
            q.put(bool(np.array_equal(full, np.stack([bx, by, bz]))))
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
