"""Multi-GPU target sharding of the tree walk.

Targets are independent once the tree exists, so N GPUs split one all-active walk by target:
every rank builds the same tree from the full particle set (the build is deterministic, so the
trees are identical and nothing is exchanged), then walks a contiguous slice of the targets in
tree order -- a Peano-Hilbert key range, hence a compact region of space -- with slice edges on
group-window boundaries so that no window is split.  The results stay on the rank that computed
them, as the engine keeps forces where the targets live; there is no collective in the data path.
Gathering the slices (for a check, or for a caller that wants all forces in one place) is a
separate, optional all-gather.
"""
from __future__ import annotations

import numpy as np


def shard_ranges(n_targets: int, world: int, window: int = 32):
    """Contiguous [start, end) slices of n_targets tree-order targets, one per rank, with every
    edge on a multiple of `window` and sizes differing by at most one window."""
    if world < 1:
        raise ValueError("world must be >= 1")
    n_win = (n_targets + window - 1) // window
    edges = [(r * n_win) // world * window for r in range(world + 1)]
    edges = [min(e, n_targets) for e in edges]
    edges[-1] = n_targets
    return [(edges[r], edges[r + 1]) for r in range(world)]


def rank_targets(orderbuf: np.ndarray, rank: int, world: int, window: int = 32) -> np.ndarray:
    """Particle indices this rank walks: its slice of orderbuf."""
    a, b = shard_ranges(len(orderbuf), world, window)[rank]
    return np.ascontiguousarray(orderbuf[a:b], np.uint32)


def gather_slices(parts, n_targets: int, world: int, window: int = 32) -> np.ndarray:
    """Reassemble per-rank result slices (in rank order) into one array over all targets."""
    out = np.empty(n_targets, dtype=np.asarray(parts[0]).dtype)
    for (a, b), p in zip(shard_ranges(n_targets, world, window), parts):
        out[a:b] = p
    return out


def walk_shard(walk, orderbuf, aold_tree, rank: int, world: int, window: int = 32):
    """This rank's part of an all-active walk of one system.

    orderbuf holds the tree order (particle indices) and aold_tree the per-target aold in the same
    order (or None).  The rank walks targets orderbuf[a:b] with aold_tree[a:b], where [a, b) is its
    window-aligned slice, so its windows are exactly the single-rank walk's windows over that
    range.  walk(targets, aold) does the walking (the GPU context, or the oracle in the CPU tests)
    and returns the results parallel to targets.  Returns (a, b, results)."""
    a, b = shard_ranges(len(orderbuf), world, window)[rank]
    tg = orderbuf[a:b]
    ao = None if aold_tree is None else aold_tree[a:b]
    return a, b, walk(tg, ao)

