"""gt_tree_audit, the device-side port of shmem::audit_tree (shmem/tree.cc:973-1119).

Freshly built trees of every kind this library builds must audit clean: Morton and Peano-Hilbert
keys, massless particles, a collocated clump that forces level-20 leaves, a randomised root, a
forest of systems, and a deep clustered box.  A tree whose particles have moved since the build
(gt_tree_particles without a refresh) must not: its nodes' centres of mass and cells no longer
describe the particles, which is what the reference's audit exists to catch.
"""
import numpy as np
import pytest

import gizmo_shared_memory_b200 as g
from gizmo_shared_memory_b200 import ics

pytestmark = pytest.mark.gpu


def clean(ctx, T):
    nb, msg = ctx.tree_audit(T)
    assert nb == 0, msg


def test_fresh_trees_audit_clean(gpu_ctx):
    P = ics.plummer(n=65536, seed=42, soft=0.01)
    for mode in (g.GT_KEY_MORTON, g.GT_KEY_PEANO):
        clean(gpu_ctx, gpu_ctx.build(P, key_mode=mode))
    clean(gpu_ctx, gpu_ctx.build(P, randomize_seed=7))
    # massless particles sort last and stay out of the tree
    Q = {k: v.copy() for k, v in P.items()}
    Q["m"][::13] = 0.0
    clean(gpu_ctx, gpu_ctx.build(Q))
    # a collocated clump: 40 particles at one point force a level-20 leaf above leaf_max
    R = {k: v[:4096].copy() for k, v in P.items()}
    R["x"][:40] = R["x"][0]
    R["y"][:40] = R["y"][0]
    R["z"][:40] = R["z"][0]
    clean(gpu_ctx, gpu_ctx.build(R))
    # a forest of three systems
    F = {k: np.concatenate([P[k][:3000], P[k][3000:9000] + (25.0 if k == "x" else 0.0), P[k][9000:20000]])
         for k in P}
    clean(gpu_ctx, gpu_ctx.build(F, offsets=np.array([0, 3000, 9000, 20000], np.int64)))
    clean(gpu_ctx, gpu_ctx.build(ics.soneira_peebles(levels=10, seed=8)))


def test_moved_particles_fail_the_audit(gpu_ctx):
    P = ics.plummer(n=20000, seed=3, soft=0.01)
    T = gpu_ctx.build(P)
    clean(gpu_ctx, T)
    moved = {k: P[k].copy() for k in ("x", "y", "z")}
    moved["x"][::50] += 5.0
    gpu_ctx.tree_particles(T, x=moved["x"], y=moved["y"], z=moved["z"])
    nb, msg = gpu_ctx.tree_audit(T)
    assert nb > 0
    assert "cell" in msg or "centre of mass" in msg, msg
