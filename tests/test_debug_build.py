"""The bounds-checked library (libgt_debug.so: the same kernels built with -DGT_BOUNDS_CHECK, the
build's stand-in for a memory checker) runs the walks clean and gives the ordinary library's
results.  It runs in a child process, since a process loads one libgt at a time: the child walks a
Plummer sphere with leaf groups, windows (two per warp), explicit targets in leaf groups and in
windows, node groups, and a forest, on both
libraries in turn (fresh contexts each), and every call must return GT_OK with identical forces."""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import os, sys
ROOT = sys.argv[1]
import numpy as np
sys.path.insert(0, ROOT)
import gizmo_shared_memory_b200 as g
from gizmo_shared_memory_b200 import _gt, ics

def run(lib):
    _gt._LIB = None
    _gt.load_library(lib)
    ctx = g.Context(0)
    P = ics.plummer(n=30000, seed=9, soft=0.01)
    T = ctx.build(P)
    ob = T.download(nodes=False)["orderbuf"]
    out = []
    a = ctx.accel_grouped(T, None, theta=0.7)
    out += list(a)
    aold = 0.003 * np.sqrt(a[0] ** 2 + a[1] ** 2 + a[2] ** 2)
    out += list(ctx.accel_grouped(T, None, aold=aold, batch=32, group_mode=g.GT_GROUP_BATCH))
    out += list(ctx.accel_grouped(T, None, aold=aold, group_mode=g.GT_GROUP_NODE, group_max=64))
    sub = ob[::7].copy()
    out += list(ctx.accel_grouped(T, sub, aold=aold[::7].copy(), batch=0))
    out += list(ctx.accel_grouped(T, sub, aold=aold[::7].copy(), batch=32, group_mode=g.GT_GROUP_BATCH))
    F = ctx.build({k: np.concatenate([v[:10000], v[10000:] + (30.0 if k == "x" else 0.0)]) for k, v in P.items()},
                  offsets=np.array([0, 10000, 30000], np.int64))
    out += list(ctx.accel_grouped(F, None, theta=0.7, batch=32, group_mode=g.GT_GROUP_BATCH))
    ctx.close()
    return out

lib = os.path.join(ROOT, "gizmo_shared_memory_b200", "lib")
dbg = run(os.path.join(lib, "libgt_debug.so"))
ref = run(os.path.join(lib, "libgt.so"))
assert len(dbg) == len(ref)
for a, b in zip(dbg, ref):
    assert np.array_equal(a, b)
print("debug library: %d outputs identical" % len(dbg))
"""


def test_bounds_checked_library_runs_clean_and_identical():
    dbg = os.path.join(ROOT, "gizmo_shared_memory_b200", "lib", "libgt_debug.so")
    if not os.path.exists(dbg):
        pytest.fail("libgt_debug.so not built (make -C gizmo_shared_memory_b200/csrc debug)")
    r = subprocess.run([sys.executable, "-c", CHILD, ROOT], capture_output=True, text=True, timeout=600)
    print(r.stdout, r.stderr[-2000:])
    assert r.returncode == 0
    assert "identical" in r.stdout
