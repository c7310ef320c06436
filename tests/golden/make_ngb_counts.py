"""Generate tests/golden/ngb_counts.npz: the reference's SHMEM_NGB_COUNT totals (shmem/hydro.cc:7-35)
on the neighbour-search fixture of golden.npz.

Runs the reference's own hydro, compiled from its sources into oracle/_ref/libgizmo_ref.so, with
SHMEM_NGB_COUNT set before its first search (the reference reads the variable once).  Records, each
from zeroed totals:

* gather: one ngb_search per centre of the fixture (its 400 centres and radii), fresh tree;
* stale: the same search on a tree built with velocities, 0.05 time units after its build, where
  the per-node vmax pad admits extra nodes (the pad-only node count), with the lists it found;
* density: the cold density solve of the fixture's gas targets (calls, nodes, examined, kept and
  the iteration histogram).

Regenerate with:

    make -C oracle ref && python tests/golden/make_ngb_counts.py
"""
import ctypes as C
import os
import sys

os.environ["SHMEM_NGB_COUNT"] = "1"

import numpy as np  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from oracle import Reference  # noqa: E402

STALE_ELAPSED = 0.05


def fixture_particles(gold):
    P = {k: np.ascontiguousarray(gold[f"ngb_{k}"]) for k in ("x", "y", "z", "m", "type")}
    P["soft"] = np.full(len(P["m"]), 0.01)
    P["zeta"] = np.zeros(len(P["m"]))
    return P


def velocities(n):
    rng = np.random.default_rng(91)
    return [rng.normal(0.0, 0.5, n) for _ in range(3)]


def one_gather_pass(R, T, cen, rad):
    """One ngb_search per centre (a count-only call of the wrapper: a single traversal each)."""
    cx, cy, cz, r = (np.ascontiguousarray(a, np.float64) for a in (*cen, rad))
    n = len(cx)
    start = np.zeros(n + 1, np.int64)
    d = C.POINTER(C.c_double)
    R.L.ref_ngb_search(T.h, n, cx.ctypes.data_as(d), cy.ctypes.data_as(d), cz.ctypes.data_as(d),
                       r.ctypes.data_as(d), 0, None, 0, 0.0, start.ctypes.data_as(C.POINTER(C.c_int64)), None, 0)
    return start


def main():
    gold = np.load(os.path.join(HERE, "golden.npz"))
    R = Reference()
    R.set_threads(4)
    P = fixture_particles(gold)
    cen = [gold[f"ngb_c{k}"] for k in "xyz"]
    rad = gold["ngb_radius"]
    out = {}

    T = R.build_gas(P)
    R.ngb_counters(reset=True)
    one_gather_pass(R, T, cen, rad)
    out["gather"] = R.ngb_counters(reset=True)

    vel = velocities(len(P["m"]))
    TV = R.build(P, vel=vel)
    TV.set_elapsed(STALE_ELAPSED)
    R.ngb_counters(reset=True)
    one_gather_pass(R, TV, cen, rad)
    out["stale"] = R.ngb_counters(reset=True)
    st, f = TV.ngb_search(*cen, rad)
    out["stale_start"], out["stale_found"] = st, f
    R.ngb_counters(reset=True)

    T.density(gold["ngb_targets"], 32.0, 0.05)
    out["density"] = R.ngb_counters(reset=True)
    out["stale_elapsed"] = np.array([STALE_ELAPSED])
    for k in ("vx", "vy", "vz"):
        out[k] = vel["xyz".index(k[1])]
    np.savez_compressed(os.path.join(HERE, "ngb_counts.npz"), **out)
    for k in ("gather", "stale", "density"):
        print(k, out[k].tolist())


if __name__ == "__main__":
    main()
