"""Multi-GPU target sharding of the tree walk.

Targets are independent once the tree exists, so N GPUs split one all-active walk by target:
every rank builds the same tree from the full particle set (the build is deterministic, so the
trees are identical and nothing is exchanged), then walks a contiguous slice of the targets in
tree order -- a Peano-Hilbert key range, hence a compact region of space -- with slice edges on
boundaries of two group windows, so that no window is split and the walk pairs windows as the
single-rank walk does.  The results stay on the rank that computed
them, as the engine keeps forces where the targets live; there is no collective in the data path.
Gathering the slices (for a check, or for a caller that wants all forces in one place) is a
separate, optional all-gather.
"""
from __future__ import annotations

import numpy as np


def shard_ranges(n_targets: int, world: int, window: int = 32):
    """Contiguous [start, end) slices of n_targets tree-order targets, one per rank, with every
    edge on a multiple of two windows and sizes differing by at most two windows.  The walk takes
    consecutive windows two per warp, pairing windows 2p and 2p + 1 of its target list; a slice
    that starts on an even window pairs its windows as the single-rank walk does, so the ranks'
    results are those of the single-rank walk bit for bit."""
    if world < 1:
        raise ValueError("world must be >= 1")
    unit = 2 * window
    n_unit = (n_targets + unit - 1) // unit
    edges = [(r * n_unit) // world * unit for r in range(world + 1)]
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
    slice (aligned to two windows), so its windows, and the pairs of windows its warps walk, are
    exactly the single-rank walk's over that range.  walk(targets, aold) does the walking (the GPU context, or the oracle in the CPU tests)
    and returns the results parallel to targets.  Returns (a, b, results)."""
    a, b = shard_ranges(len(orderbuf), world, window)[rank]
    tg = orderbuf[a:b]
    ao = None if aold_tree is None else aold_tree[a:b]
    return a, b, walk(tg, ao)

