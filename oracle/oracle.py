"""ORACLE — test infrastructure only.

ctypes bindings for the two CPU checkers of the tree-gravity path:

* ``Restatement`` loads ``oracle/liboracle.so``: the plain-C restatement in ``gt_oracle.c``
  (each function cites the reference file:line it follows).
* ``Reference`` loads ``oracle/_ref/libgizmo_ref.so``: the reference's own ``shmem/tree.cc`` and
  Peano-Hilbert functions, compiled from the reference sources by ``oracle/Makefile`` (target
  ``ref``).  It is absent wherever the reference sources were not available at build time.

Only ``tests/``, ``bench.py``'s CPU-baseline leg / reference arm and ``__graft_entry__.smoke()``
import this module, and only as the checker or the timed CPU baseline; the product library never
calls into it.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
RESTATEMENT_SO = os.path.join(HERE, "liboracle.so")
REFERENCE_SO = os.path.join(HERE, "_ref", "libgizmo_ref.so")

_d = C.POINTER(C.c_double)
_f = C.POINTER(C.c_float)
_i = C.POINTER(C.c_int)
_u32 = C.POINTER(C.c_uint32)
_u64 = C.POINTER(C.c_uint64)
_i64 = C.POINTER(C.c_int64)


def _p(a, ctype):
    if a is None:
        return None
    return a.ctypes.data_as(ctype)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _targets(t):
    return np.ascontiguousarray(t, dtype=np.uint32)


def build_library():
    """Compile liboracle.so (and _ref when the reference sources are present)."""
    import subprocess

    subprocess.run(["make", "-s", "-C", HERE], check=True)
    # the recipe finds the reference sources ($GIZMO_REF) and skips _ref where they are absent
    subprocess.run(["make", "-s", "-C", HERE, "ref-if-present"], check=True)


def reference_available() -> bool:
    return os.path.exists(REFERENCE_SO)


class Restatement:
    """The plain-C restatement (gt_oracle.c)."""

    def __init__(self, path: str = RESTATEMENT_SO):
        if not os.path.exists(path):
            build_library()
        L = C.CDLL(path)
        self.L = L
        L.or_spline_force_over_r.restype = C.c_double
        L.or_spline_force_over_r.argtypes = [C.c_double, C.c_double]
        L.or_spline_potential.restype = C.c_double
        L.or_spline_potential.argtypes = [C.c_double, C.c_double]
        L.or_open_node.restype = C.c_int
        L.or_open_node.argtypes = [C.c_double] * 11
        L.or_morton20.restype = C.c_uint64
        L.or_morton20.argtypes = [C.c_uint32] * 3
        L.or_peano_key.argtypes = [C.c_uint64] * 3 + [C.c_int, _u64, _u64]
        L.or_morton_key.argtypes = [C.c_uint64] * 3 + [C.c_int, _u64, _u64]
        L.or_double_to_int.restype = C.c_uint64
        L.or_double_to_int.argtypes = [C.c_double, C.c_int]
        L.or_keys20.argtypes = [C.c_int64, _d, _d, _d, _d, C.c_int, C.c_longlong, _u64, _d]
        L.or_build.restype = C.c_void_p
        L.or_build.argtypes = [C.c_int64, _d, _d, _d, _d, _d, C.c_longlong, C.c_int]
        L.or_free.argtypes = [C.c_void_p]
        L.or_nnodes.restype = C.c_int64
        L.or_nnodes.argtypes = [C.c_void_p]
        L.or_nlive.restype = C.c_int64
        L.or_nlive.argtypes = [C.c_void_p]
        L.or_root.restype = C.c_int
        L.or_root.argtypes = [C.c_void_p]
        L.or_nodes.argtypes = [C.c_void_p] + [_d] * 10 + [_i] * 6 + [_d, _f, _f]
        L.or_order.argtypes = [C.c_void_p, _u32, _u32, _i]
        L.or_groups.restype = C.c_int64
        L.or_groups.argtypes = [C.c_void_p, C.c_int64, _u32, C.c_int, _i64]
        L.or_walk_groups.argtypes = [C.c_void_p, C.c_int64, _u32, C.c_int64, _i64, C.c_double,
                                     C.c_double, _d, C.c_int, _d, _d, _d, _d, _i64]
        L.or_accel_grouped.argtypes = [C.c_void_p, C.c_int64, _u32, C.c_double, C.c_double,
                                       C.c_int, _d, _d, _d, _d, _i64]
        L.or_accel.argtypes = [C.c_void_p, C.c_int64, _u32, C.c_double, C.c_double, _d, _d, _d, _d]
        L.or_potential.argtypes = [C.c_void_p, C.c_int64, _u32, C.c_double, C.c_double, _d, _d]
        L.or_set_walk_nodes.argtypes = [C.c_void_p, _d, _d, _d, _d, _d, _f, _f]
        L.or_set_positions.argtypes = [C.c_void_p, _d, _d, _d]
        L.or_spline_tidal_factor.restype = C.c_double
        L.or_spline_tidal_factor.argtypes = [C.c_double, C.c_double]
        L.or_velocity_moments.argtypes = [C.c_void_p, _d, _d, _d, _d, _d, _d, _f]
        L.or_walk_groups_ext.argtypes = [C.c_void_p, C.c_int64, _u32, C.c_int64, _i64, C.c_double,
                                         C.c_double, _d] + [_d] * 11
        L.or_direct.argtypes = [C.c_int64, _d, _d, _d, _d, _d, C.c_int64, _u32, C.c_double,
                                _d, _d, _d, _d]
        L.or_kernel_dwdr.restype = C.c_double
        L.or_kernel_dwdr.argtypes = [C.c_double, C.c_double]
        L.or_walk_groups_gas.argtypes = [C.c_void_p, C.c_int64, _u32, C.c_int64, _i64, C.c_double,
                                         C.c_double, _d, C.c_void_p, _d, C.c_double, C.c_int, _d, _d, _d]
        L.or_node_sinks.argtypes = [C.c_void_p, C.c_void_p, _u32]
        L.or_direct_gas.argtypes = [C.c_int64, _d, _d, _d, _d, _d, C.c_void_p, _d, C.c_int64, _u32, C.c_double,
                                    _d, _d, _d]
        L.or_ngb_search.argtypes = [C.c_void_p, C.c_int64, _d, _d, _d, _d, C.c_int, _d, C.c_int64, C.c_double,
                                    _i64, _u32, C.c_int64]
        L.or_init_hmax.argtypes = [C.c_void_p, _d, C.c_int64, _f]
        L.or_density.argtypes = [C.c_void_p, C.c_int64, _u32, C.c_double, C.c_double, _d, C.c_double, C.c_int, _d,
                                 C.c_void_p, C.c_int, _d, _d, C.c_void_p, C.c_void_p]

    # scalar helpers
    def spline_force_over_r(self, r, h):
        return self.L.or_spline_force_over_r(r, h)

    def spline_potential(self, r, h):
        return self.L.or_spline_potential(r, h)

    def open_node(self, *args):
        return self.L.or_open_node(*[float(a) for a in args])

    def peano_key(self, x, y, z, bits):
        hi, lo = C.c_uint64(), C.c_uint64()
        self.L.or_peano_key(int(x), int(y), int(z), bits, C.byref(hi), C.byref(lo))
        return (hi.value << 64) | lo.value

    def morton_key(self, x, y, z, bits):
        hi, lo = C.c_uint64(), C.c_uint64()
        self.L.or_morton_key(int(x), int(y), int(z), bits, C.byref(hi), C.byref(lo))
        return (hi.value << 64) | lo.value

    def morton20(self, a, b, c):
        return self.L.or_morton20(int(a), int(b), int(c))

    def double_to_int(self, d, bits=42):
        return self.L.or_double_to_int(float(d), bits)

    def keys20(self, P, key_mode=1, randomize_seed=-1):
        n = len(P["m"])
        keys = np.empty(n, np.uint64)
        geom = np.empty(5, np.float64)
        x, y, z, m = (_f64(P[k]) for k in ("x", "y", "z", "m"))
        self.L.or_keys20(n, _p(x, _d), _p(y, _d), _p(z, _d), _p(m, _d), key_mode, randomize_seed,
                         _p(keys, _u64), _p(geom, _d))
        return keys, geom

    def build(self, P, randomize_seed=-1, nodelta=False):
        return OracleTree(self, P, randomize_seed, nodelta)

    def direct_gas(self, P, targets, type=None, zeta=None, G=1.0):
        """accel_brute with the gas pair rule: FP64 direct sum with the zeta terms."""
        x, y, z, m = (_f64(P[k]) for k in ("x", "y", "z", "m"))
        soft = _f64(P["soft"]) if P.get("soft") is not None else None
        ty = None if type is None else np.ascontiguousarray(type, np.uint8)
        ze = None if zeta is None else _f64(zeta)
        t = _targets(targets)
        nt = len(t)
        ax, ay, az = np.empty(nt), np.empty(nt), np.empty(nt)
        self.L.or_direct_gas(len(m), _p(x, _d), _p(y, _d), _p(z, _d), _p(m, _d), _p(soft, _d),
                             None if ty is None else ty.ctypes.data, _p(ze, _d), nt, _p(t, _u32), G,
                             _p(ax, _d), _p(ay, _d), _p(az, _d))
        return ax, ay, az

    def direct(self, P, targets, G=1.0, want_phi=True):
        t = _targets(targets)
        nt = len(t)
        ax, ay, az = np.empty(nt), np.empty(nt), np.empty(nt)
        phi = np.empty(nt) if want_phi else None
        x, y, z, m = (_f64(P[k]) for k in ("x", "y", "z", "m"))
        soft = _f64(P["soft"]) if P.get("soft") is not None else None
        self.L.or_direct(len(m), _p(x, _d), _p(y, _d), _p(z, _d), _p(m, _d), _p(soft, _d), nt,
                         _p(t, _u32), G, _p(ax, _d), _p(ay, _d), _p(az, _d), _p(phi, _d))
        return (ax, ay, az, phi) if want_phi else (ax, ay, az)


class OracleTree:
    """A restatement tree; keeps the particle arrays it borrows alive."""

    def __init__(self, lib: Restatement, P, randomize_seed=-1, nodelta=False):
        self.lib = lib
        self._keep = [_f64(P[k]) for k in ("x", "y", "z", "m")]
        soft = P.get("soft")
        self._soft = _f64(soft) if soft is not None else None
        x, y, z, m = self._keep
        self.n = len(m)
        self.h = lib.L.or_build(self.n, _p(x, _d), _p(y, _d), _p(z, _d), _p(m, _d),
                                _p(self._soft, _d), randomize_seed, int(nodelta))

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.L.or_free(self.h)
            self.h = None

    @property
    def nnodes(self):
        return self.lib.L.or_nnodes(self.h)

    @property
    def nlive(self):
        return self.lib.L.or_nlive(self.h)

    @property
    def root(self):
        return self.lib.L.or_root(self.h)

    def nodes(self):
        nn = self.nnodes
        out = {k: np.empty(nn) for k in ("cx", "cy", "cz", "mass", "size", "delta", "soft", "gcx",
                                           "gcy", "gcz")}
        for k in ("first", "next", "plo", "phi", "parent", "level"):
            out[k] = np.empty(nn, np.int32)
        out["w_s"] = np.empty(nn)
        out["w_len"] = np.empty(nn, np.float32)
        out["w_soft"] = np.empty(nn, np.float32)
        L = self.lib.L
        L.or_nodes(self.h, *[_p(out[k], _d) for k in ("cx", "cy", "cz", "mass", "size", "delta",
                                                        "soft", "gcx", "gcy", "gcz")],
                   *[_p(out[k], _i) for k in ("first", "next", "plo", "phi", "parent", "level")],
                   _p(out["w_s"], _d), _p(out["w_len"], _f), _p(out["w_soft"], _f))
        return out

    def order(self):
        ob = np.empty(self.nlive, np.uint32)
        rank = np.empty(self.n, np.uint32)
        leaf = np.empty(self.n, np.int32)
        self.lib.L.or_order(self.h, _p(ob, _u32), _p(rank, _u32), _p(leaf, _i))
        return ob, rank, leaf

    def groups(self, targets, batch=0):
        t = _targets(targets)
        starts = np.empty(len(t) + 1, np.int64)
        ng = self.lib.L.or_groups(self.h, len(t), _p(t, _u32), batch, _p(starts, _i64))
        return starts[: ng + 1].copy()

    def walk_groups(self, targets, starts, theta, G=1.0, aold=None, leaf_accept=True,
                    want_phi=False):
        t = _targets(targets)
        nt = len(t)
        st = np.ascontiguousarray(starts, np.int64)
        ax, ay, az = np.empty(nt), np.empty(nt), np.empty(nt)
        phi = np.empty(nt) if want_phi else None
        cnt = np.zeros(3, np.int64)
        ao = _f64(aold) if aold is not None else None
        self.lib.L.or_walk_groups(self.h, nt, _p(t, _u32), len(st) - 1, _p(st, _i64), theta, G,
                                  _p(ao, _d), int(leaf_accept), _p(ax, _d), _p(ay, _d),
                                  _p(az, _d), _p(phi, _d), _p(cnt, _i64))
        return ax, ay, az, phi, cnt

    def set_walk_nodes(self, st):
        """Overwrite the walk's node fields with refreshed ones (oracle.reuse.Reuse.refresh)."""
        self._walk_nodes = [np.ascontiguousarray(st["com"][:, k], np.float64) for k in range(3)] + [
            _f64(st["mass"]), _f64(st["w_s"]), np.ascontiguousarray(st["w_len"], np.float32),
            np.ascontiguousarray(st["w_soft"], np.float32)]
        cx, cy, cz, m, s, ln, sf = self._walk_nodes
        self.lib.L.or_set_walk_nodes(self.h, _p(cx, _d), _p(cy, _d), _p(cz, _d), _p(m, _d), _p(s, _d),
                                     _p(ln, _f), _p(sf, _f))

    def set_positions(self, x, y, z):
        self._pos = [_f64(a) for a in (x, y, z)]
        self.lib.L.or_set_positions(self.h, *[_p(a, _d) for a in self._pos])

    def velocity_moments(self, vel):
        """Node centre-of-mass velocity (3 arrays) and speed bound for velocities vel = (vx, vy, vz)."""
        v = [_f64(a) for a in vel]
        nn = self.nnodes
        vc = [np.zeros(nn) for _ in range(3)]
        vmax = np.zeros(nn, np.float32)
        self.lib.L.or_velocity_moments(self.h, _p(v[0], _d), _p(v[1], _d), _p(v[2], _d), _p(vc[0], _d),
                                       _p(vc[1], _d), _p(vc[2], _d), _p(vmax, _f))
        return vc, vmax

    def walk_groups_ext(self, targets, starts, theta, G=1.0, aold=None, vel=None, tidal=True):
        """Grouped walk with the tidal tensor ([nt, 6], not times G) and, given vel, the jerk ([nt, 3])."""
        t = _targets(targets)
        nt = len(t)
        st = np.ascontiguousarray(starts, np.int64)
        ax, ay, az = np.empty(nt), np.empty(nt), np.empty(nt)
        tt = np.zeros((nt, 6)) if tidal else None
        jj = None
        v = vc = [None, None, None]
        if vel is not None:
            v = [_f64(a) for a in vel]
            vc, _ = self.velocity_moments(v)
            jj = np.zeros((nt, 3))
        ao = _f64(aold) if aold is not None else None
        self.lib.L.or_walk_groups_ext(self.h, nt, _p(t, _u32), len(st) - 1, _p(st, _i64), theta, G, _p(ao, _d),
                                      *[_p(a, _d) for a in v], *[_p(a, _d) for a in vc], _p(ax, _d), _p(ay, _d),
                                      _p(az, _d), _p(tt, _d), _p(jj, _d))
        return ax, ay, az, tt, jj

    def walk_groups_gas(self, targets, starts, theta, G=1.0, aold=None, type=None, zeta=None,
                        sink_radius=0.0, leaf_accept=True):
        """Walk with the gas pair rule (zeta terms for gas-gas pairs) and, grouped, sink-direct
        opening; type (uint8, 0 gas, 5 sink) and zeta are indexed like the build's particles."""
        t = _targets(targets)
        nt = len(t)
        st = np.ascontiguousarray(starts, np.int64)
        ax, ay, az = np.empty(nt), np.empty(nt), np.empty(nt)
        ty = None if type is None else np.ascontiguousarray(type, np.uint8)
        ze = None if zeta is None else _f64(zeta)
        ao = _f64(aold) if aold is not None else None
        self.lib.L.or_walk_groups_gas(self.h, nt, _p(t, _u32), len(st) - 1, _p(st, _i64), theta, G, _p(ao, _d),
                                      None if ty is None else ty.ctypes.data, _p(ze, _d), sink_radius,
                                      int(leaf_accept), _p(ax, _d), _p(ay, _d), _p(az, _d))
        return ax, ay, az

    def ngb_search(self, cx, cy, cz, radius, mode=0, h=None, n_gas=0, box=0.0):
        """Neighbour lists (start [n+1], found) in tree order: mode 0 gather, 1 reverse, 2 both."""
        cx, cy, cz, r = (_f64(a) for a in (cx, cy, cz, radius))
        n = len(cx)
        hv = _f64(h) if h is not None else None
        start = np.zeros(n + 1, np.int64)
        self.lib.L.or_ngb_search(self.h, n, _p(cx, _d), _p(cy, _d), _p(cz, _d), _p(r, _d), mode, _p(hv, _d),
                                 int(n_gas), box, _p(start, _i64), None, 0)
        found = np.zeros(max(int(start[-1]), 1), np.uint32)
        self.lib.L.or_ngb_search(self.h, n, _p(cx, _d), _p(cy, _d), _p(cz, _d), _p(r, _d), mode, _p(hv, _d),
                                 int(n_gas), box, _p(start, _i64), _p(found, _u32), len(found))
        return start, found[: start[-1]]

    def init_hmax(self, h, n_gas):
        hv = _f64(h)
        out = np.zeros(self.nnodes, np.float32)
        self.lib.L.or_init_hmax(self.h, _p(hv, _d), int(n_gas), _p(out, _f))
        return out

    def density(self, targets, des_ngb=32.0, ngb_tol=0.05, h_start=None, box=0.0, n_dims=3, cond_prev=None,
                type=None, face_corr=True):
        t = _targets(targets)
        nt = len(t)
        h, rho = np.zeros(nt), np.zeros(nt)
        nngb, iters = np.zeros(nt, np.int32), np.zeros(nt, np.int32)
        hs = _f64(h_start) if h_start is not None else None
        cp = _f64(cond_prev) if cond_prev is not None else None
        ty = None if type is None else np.ascontiguousarray(type, np.uint8)
        self.lib.L.or_density(self.h, nt, _p(t, _u32), des_ngb, ngb_tol, _p(hs, _d), box, n_dims, _p(cp, _d),
                              None if ty is None else ty.ctypes.data, int(face_corr), _p(h, _d), _p(rho, _d),
                              nngb.ctypes.data, iters.ctypes.data)
        return {"h": h, "rho": rho, "nngb": nngb, "iters": iters}

    def node_sinks(self, type):
        ty = np.ascontiguousarray(type, np.uint8)
        out = np.zeros(self.nnodes, np.uint32)
        self.lib.L.or_node_sinks(self.h, ty.ctypes.data, _p(out, _u32))
        return out

    def accel_grouped(self, targets, theta, G=1.0, batch=0, aold=None):
        t = _targets(targets)
        nt = len(t)
        ax, ay, az = np.empty(nt), np.empty(nt), np.empty(nt)
        cnt = np.zeros(3, np.int64)
        ao = _f64(aold) if aold is not None else None
        self.lib.L.or_accel_grouped(self.h, nt, _p(t, _u32), theta, G, batch, _p(ao, _d),
                                    _p(ax, _d), _p(ay, _d), _p(az, _d), _p(cnt, _i64))
        return ax, ay, az, cnt

    def accel(self, targets, theta, G=1.0, aold=None):
        t = _targets(targets)
        nt = len(t)
        ax, ay, az = np.empty(nt), np.empty(nt), np.empty(nt)
        ao = _f64(aold) if aold is not None else None
        self.lib.L.or_accel(self.h, nt, _p(t, _u32), theta, G, _p(ao, _d), _p(ax, _d), _p(ay, _d),
                            _p(az, _d))
        return ax, ay, az

    def potential(self, targets, theta, G=1.0, aold=None):
        t = _targets(targets)
        phi = np.empty(len(t))
        ao = _f64(aold) if aold is not None else None
        self.lib.L.or_potential(self.h, len(t), _p(t, _u32), theta, G, _p(ao, _d), _p(phi, _d))
        return phi


class Reference:
    """The reference's own shmem tree, compiled from its sources into oracle/_ref."""

    def __init__(self, path: str = REFERENCE_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} not built (reference sources unavailable)")
        L = C.CDLL(path)
        self.L = L
        L.ref_max_threads.restype = C.c_int
        L.ref_set_threads.argtypes = [C.c_int]
        L.ref_build.restype = C.c_void_p
        L.ref_build.argtypes = [C.c_int64, _d, _d, _d, _d, _d, C.c_longlong, _d]
        L.ref_free.argtypes = [C.c_void_p]
        L.ref_tree_nnodes.restype = C.c_int64
        L.ref_tree_nnodes.argtypes = [C.c_void_p]
        L.ref_tree_root.restype = C.c_int
        L.ref_tree_root.argtypes = [C.c_void_p]
        L.ref_tree_nlive.restype = C.c_int64
        L.ref_tree_nlive.argtypes = [C.c_void_p]
        L.ref_tree_nodes.argtypes = [C.c_void_p] + [_d] * 10 + [_i] * 5 + [_d, _f, _f]
        L.ref_tree_order.argtypes = [C.c_void_p, _u32, _u32, _i]
        L.ref_accel_grouped.argtypes = [C.c_void_p, C.c_int64, _u32, C.c_double, C.c_double,
                                        C.c_int, _d, _d, _d, _d]
        L.ref_accel.argtypes = [C.c_void_p, C.c_int64, _u32, C.c_double, C.c_double, _d, _d, _d, _d]
        L.ref_potential.argtypes = [C.c_void_p, C.c_int64, _u32, C.c_double, C.c_double, _d, _d]
        L.ref_accel_brute.argtypes = [C.c_void_p, C.c_int64, _u32, C.c_double, _d, _d, _d]
        L.ref_morton20.restype = C.c_uint64
        L.ref_morton20.argtypes = [C.c_uint32] * 3
        L.ref_peano_hilbert_key.argtypes = [C.c_uint64] * 3 + [C.c_int, _u64, _u64]
        L.ref_morton_key.argtypes = [C.c_uint64] * 3 + [C.c_int, _u64, _u64]
        L.ref_peano_and_morton_key.argtypes = [C.c_uint64] * 3 + [C.c_int, _u64, _u64, _u64, _u64]
        L.ref_domain_double_to_int.restype = C.c_uint64
        L.ref_domain_double_to_int.argtypes = [C.c_double]
        L.ref_spline_force_over_r.restype = C.c_double
        L.ref_spline_force_over_r.argtypes = [C.c_double, C.c_double]
        L.ref_spline_potential.restype = C.c_double
        L.ref_spline_potential.argtypes = [C.c_double, C.c_double]
        L.ref_open_node.restype = C.c_int
        L.ref_open_node.argtypes = [C.c_double] * 11
        L.ref_build_vel.restype = C.c_void_p
        L.ref_build_vel.argtypes = [C.c_int64] + [_d] * 8 + [C.c_longlong]
        L.ref_tree_vel.argtypes = [C.c_void_p, _d, _d, _d, _f]
        L.ref_accel_grouped_ext.argtypes = [C.c_void_p, C.c_int64, _u32, C.c_double, C.c_double,
                                            C.c_int, _d, _d, _d, _d, _d, _d]
        L.ref_build_gas.restype = C.c_void_p
        L.ref_build_gas.argtypes = [C.c_int64] + [_d] * 6 + [C.c_void_p]
        L.ref_accel_grouped_gas.argtypes = [C.c_void_p, C.c_int64, _u32, C.c_double, C.c_double, C.c_int, _d,
                                            C.c_double, _d, _d, _d]
        L.ref_tree_nsink.argtypes = [C.c_void_p, _u32]
        L.ref_set_elapsed.argtypes = [C.c_void_p, C.c_double]
        L.ref_ngb_counters.argtypes = [_i64, C.c_int]
        L.ref_init_hmax.argtypes = [C.c_void_p, _d, C.c_int64, _f]
        L.ref_raise_hmax.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, _d]
        L.ref_ngb_search.argtypes = [C.c_void_p, C.c_int64, _d, _d, _d, _d, C.c_int, _d, C.c_int64, C.c_double,
                                     _i64, _u32, C.c_int64]
        L.ref_density.argtypes = [C.c_void_p, C.c_int64, _u32, C.c_double, C.c_double, _d, C.c_double, C.c_int, _d,
                                  _d, _d, C.c_void_p, C.c_void_p, _i64, _u32, C.c_int64]
        L.ref_reuse_begin.argtypes = [C.c_void_p]
        L.ref_kick_node.argtypes = [C.c_void_p, C.c_int, _d, C.c_double]
        L.ref_mass_event.argtypes = [C.c_void_p, C.c_int, C.c_double, _d, _d, C.c_double, C.c_double]
        L.ref_shift_node.argtypes = [C.c_void_p, C.c_int, C.c_double, _d]
        L.ref_raise_vmax.argtypes = [C.c_void_p, C.c_int, C.c_float]
        L.ref_raise_pad.argtypes = [C.c_void_p, C.c_int, C.c_double]
        L.ref_raise_soft.argtypes = [C.c_void_p, C.c_int, C.c_double]
        L.ref_refresh_walk_nodes.argtypes = [C.c_void_p, C.c_double]
        L.ref_node_state.argtypes = [C.c_void_p, C.c_double, _d, _d, _d, _f, _f, _d, _f, _f]
        L.ref_set_positions.argtypes = [C.c_void_p, _d, _d, _d]

    def max_threads(self):
        return self.L.ref_max_threads()

    def set_threads(self, n):
        self.L.ref_set_threads(int(n))

    def peano_key(self, x, y, z, bits):
        hi, lo = C.c_uint64(), C.c_uint64()
        self.L.ref_peano_hilbert_key(int(x), int(y), int(z), bits, C.byref(hi), C.byref(lo))
        return (hi.value << 64) | lo.value

    def morton_key(self, x, y, z, bits):
        hi, lo = C.c_uint64(), C.c_uint64()
        self.L.ref_morton_key(int(x), int(y), int(z), bits, C.byref(hi), C.byref(lo))
        return (hi.value << 64) | lo.value

    def peano_and_morton_key(self, x, y, z, bits):
        a, b, c, d = C.c_uint64(), C.c_uint64(), C.c_uint64(), C.c_uint64()
        self.L.ref_peano_and_morton_key(int(x), int(y), int(z), bits, C.byref(a), C.byref(b),
                                        C.byref(c), C.byref(d))
        return (a.value << 64) | b.value, (c.value << 64) | d.value

    def morton20(self, a, b, c):
        return self.L.ref_morton20(int(a), int(b), int(c))

    def double_to_int(self, d):
        return self.L.ref_domain_double_to_int(float(d))

    def spline_force_over_r(self, r, h):
        return self.L.ref_spline_force_over_r(r, h)

    def spline_potential(self, r, h):
        return self.L.ref_spline_potential(r, h)

    def open_node(self, *args):
        return self.L.ref_open_node(*[float(a) for a in args])

    def build(self, P, randomize_seed=-1, vel=None):
        """vel = (vx, vy, vz): build with velocities (per-node vcom and vmax, for the jerk)."""
        return ReferenceTree(self, P, randomize_seed, vel)

    def ngb_counters(self, reset=False):
        """The reference's SHMEM_NGB_COUNT totals (13 int64: calls, nodes, examined, kept, pad
        nodes, iteration histogram[8]); zeros unless SHMEM_NGB_COUNT was set before the first search."""
        v = np.zeros(13, np.int64)
        self.L.ref_ngb_counters(_p(v, _i64), int(bool(reset)))
        return v

    def build_gas(self, P):
        """Build with P["type"] (uint8, GIZMO numbering) and P["zeta"] (adaptive-softening terms)."""
        return ReferenceTree(self, P, gas=True)


class ReferenceTree:
    def __init__(self, lib: Reference, P, randomize_seed=-1, vel=None, gas=False):
        self.lib = lib
        x, y, z, m = (_f64(P[k]) for k in ("x", "y", "z", "m"))
        soft = P.get("soft")
        soft = _f64(soft) if soft is not None else None
        self.n = len(m)
        self.build_times = np.zeros(7)
        if gas:
            self._zeta = _f64(P["zeta"])
            self._type = np.ascontiguousarray(P["type"], np.uint8)
            self.h = lib.L.ref_build_gas(self.n, _p(x, _d), _p(y, _d), _p(z, _d), _p(m, _d), _p(soft, _d),
                                         _p(self._zeta, _d), self._type.ctypes.data)
        elif vel is None:
            self.h = lib.L.ref_build(self.n, _p(x, _d), _p(y, _d), _p(z, _d), _p(m, _d), _p(soft, _d),
                                     randomize_seed, _p(self.build_times, _d))
        else:
            v = [_f64(a) for a in vel]
            self.h = lib.L.ref_build_vel(self.n, _p(x, _d), _p(y, _d), _p(z, _d), _p(m, _d), _p(soft, _d),
                                         _p(v[0], _d), _p(v[1], _d), _p(v[2], _d), randomize_seed)

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.L.ref_free(self.h)
            self.h = None

    @property
    def nnodes(self):
        return self.lib.L.ref_tree_nnodes(self.h)

    @property
    def nlive(self):
        return self.lib.L.ref_tree_nlive(self.h)

    @property
    def root(self):
        return self.lib.L.ref_tree_root(self.h)

    def nodes(self):
        nn = self.nnodes
        out = {k: np.empty(nn) for k in ("cx", "cy", "cz", "mass", "size", "delta", "soft", "gcx",
                                           "gcy", "gcz")}
        for k in ("first", "next", "plo", "phi", "parent"):
            out[k] = np.empty(nn, np.int32)
        out["w_s"] = np.empty(nn)
        out["w_len"] = np.empty(nn, np.float32)
        out["w_soft"] = np.empty(nn, np.float32)
        self.lib.L.ref_tree_nodes(self.h, *[_p(out[k], _d) for k in (
            "cx", "cy", "cz", "mass", "size", "delta", "soft", "gcx", "gcy", "gcz")],
            *[_p(out[k], _i) for k in ("first", "next", "plo", "phi", "parent")],
            _p(out["w_s"], _d), _p(out["w_len"], _f), _p(out["w_soft"], _f))
        return out

    def order(self):
        ob = np.empty(self.nlive, np.uint32)
        rank = np.empty(self.n, np.uint32)
        leaf = np.empty(self.n, np.int32)
        self.lib.L.ref_tree_order(self.h, _p(ob, _u32), _p(rank, _u32), _p(leaf, _i))
        return ob, rank, leaf

    def accel_grouped(self, targets, theta, G=1.0, batch=0, aold=None):
        t = _targets(targets)
        nt = len(t)
        ax, ay, az = np.empty(nt), np.empty(nt), np.empty(nt)
        ao = _f64(aold) if aold is not None else None
        self.lib.L.ref_accel_grouped(self.h, nt, _p(t, _u32), theta, G, batch, _p(ao, _d),
                                     _p(ax, _d), _p(ay, _d), _p(az, _d))
        return ax, ay, az

    def accel_brute(self, targets, G=1.0):
        """shmem::accel_brute (tree.cc:946-971): the FP64 direct sum over the tree's particles."""
        t = _targets(targets)
        nt = len(t)
        ax, ay, az = np.empty(nt), np.empty(nt), np.empty(nt)
        self.lib.L.ref_accel_brute(self.h, nt, _p(t, _u32), G, _p(ax, _d), _p(ay, _d), _p(az, _d))
        return ax, ay, az

    def accel_grouped_ext(self, targets, theta, G=1.0, batch=0, aold=None, tidal=True, jerk=False):
        """accel_grouped with the tidal tensor ([nt, 6]: xx yy zz xy yz xz, not times G) and the
        jerk ([nt, 3], times G; the tree must have been built with velocities)."""
        t = _targets(targets)
        nt = len(t)
        ax, ay, az = np.empty(nt), np.empty(nt), np.empty(nt)
        tt = np.empty((nt, 6)) if tidal else None
        jj = np.empty((nt, 3)) if jerk else None
        ao = _f64(aold) if aold is not None else None
        self.lib.L.ref_accel_grouped_ext(self.h, nt, _p(t, _u32), theta, G, batch, _p(ao, _d), _p(ax, _d),
                                         _p(ay, _d), _p(az, _d), _p(tt, _d), _p(jj, _d))
        return ax, ay, az, tt, jj

    # ---- tree reuse (tree.cc:211-274): events on leaf nodes of this tree's numbering ----------
    def reuse_begin(self):
        self.lib.L.ref_reuse_begin(self.h)

    def events(self, kind, leaf, a=None, x=None, v=None, f=None, tau=0.0, box=0.0):
        """Apply events of one kind in order (kinds as GT_EVENT_*: 0 kick, 1 shift, 2 vmax, 3 soft,
        4 mass, 5 pad), each with the reference's own per-event call."""
        L = self.lib.L
        for e, lf in enumerate(np.asarray(leaf)):
            lf = int(lf)
            if kind == 0:
                L.ref_kick_node(self.h, lf, _p(_f64(a[e]), _d), tau)
            elif kind == 1:
                L.ref_shift_node(self.h, lf, float(a[e]), _p(_f64(x[e]), _d))
            elif kind == 2:
                L.ref_raise_vmax(self.h, lf, float(f[e]))
            elif kind == 3:
                L.ref_raise_soft(self.h, lf, float(a[e]))
            elif kind == 4:
                L.ref_mass_event(self.h, lf, float(a[e]), _p(_f64(x[e]), _d), _p(_f64(v[e]), _d), tau, box)
            elif kind == 5:
                L.ref_raise_pad(self.h, lf, float(a[e]))

    def refresh(self, tau):
        self.lib.L.ref_refresh_walk_nodes(self.h, tau)

    def node_state(self, tau):
        nn = self.nnodes
        out = {"com": np.zeros((nn, 3)), "vel": np.zeros((nn, 3)), "mass": np.zeros(nn),
               "vmax": np.zeros(nn, np.float32), "xpad": np.zeros(nn, np.float32), "w_s": np.zeros(nn),
               "w_len": np.zeros(nn, np.float32), "w_soft": np.zeros(nn, np.float32)}
        self.lib.L.ref_node_state(self.h, tau, _p(out["com"], _d), _p(out["vel"], _d), _p(out["mass"], _d),
                                  _p(out["vmax"], _f), _p(out["xpad"], _f), _p(out["w_s"], _d),
                                  _p(out["w_len"], _f), _p(out["w_soft"], _f))
        return out

    def set_positions(self, x, y, z):
        x, y, z = (_f64(a) for a in (x, y, z))
        self.lib.L.ref_set_positions(self.h, _p(x, _d), _p(y, _d), _p(z, _d))

    def accel_grouped_gas(self, targets, theta, G=1.0, batch=0, aold=None, sink_radius=0.0):
        t = _targets(targets)
        nt = len(t)
        ax, ay, az = np.empty(nt), np.empty(nt), np.empty(nt)
        ao = _f64(aold) if aold is not None else None
        self.lib.L.ref_accel_grouped_gas(self.h, nt, _p(t, _u32), theta, G, batch, _p(ao, _d), sink_radius,
                                         _p(ax, _d), _p(ay, _d), _p(az, _d))
        return ax, ay, az

    def nsink(self):
        out = np.zeros(self.nnodes, np.uint32)
        self.lib.L.ref_tree_nsink(self.h, _p(out, _u32))
        return out

    # ---- neighbour search and the density solve (shmem/hydro.cc) ----
    def set_elapsed(self, elapsed):
        self.lib.L.ref_set_elapsed(self.h, float(elapsed))

    def init_hmax(self, h, n_gas):
        self._hmax_h = _f64(h)
        out = np.zeros(self.nnodes, np.float32)
        self.lib.L.ref_init_hmax(self.h, _p(self._hmax_h, _d), int(n_gas), _p(out, _f))
        return out

    def raise_hmax(self, leaf, h):
        lf = np.ascontiguousarray(leaf, np.int32)
        hv = _f64(h)
        self.lib.L.ref_raise_hmax(self.h, len(lf), lf.ctypes.data, _p(hv, _d))

    def ngb_search(self, cx, cy, cz, radius, mode=0, h=None, n_gas=0, box=0.0):
        """Neighbour lists (start [n+1], found) of ngb_search (mode 0), ngb_search_reverse
        (mode 1, h_i = radius, needs init_hmax) or both (mode 2), in the reference's order."""
        cx, cy, cz, r = (_f64(a) for a in (cx, cy, cz, radius))
        n = len(cx)
        hv = _f64(h) if h is not None else None
        start = np.zeros(n + 1, np.int64)
        self.lib.L.ref_ngb_search(self.h, n, _p(cx, _d), _p(cy, _d), _p(cz, _d), _p(r, _d), mode, _p(hv, _d),
                                  int(n_gas), box, _p(start, _i64), None, 0)
        found = np.zeros(max(int(start[-1]), 1), np.uint32)
        self.lib.L.ref_ngb_search(self.h, n, _p(cx, _d), _p(cy, _d), _p(cz, _d), _p(r, _d), mode, _p(hv, _d),
                                  int(n_gas), box, _p(start, _i64), _p(found, _u32), len(found))
        return start, found[: start[-1]]

    def density(self, targets, des_ngb=32.0, ngb_tol=0.05, h_start=None, box=0.0, n_dims=3, cond_prev=None,
                cache=False):
        t = _targets(targets)
        nt = len(t)
        h, rho = np.zeros(nt), np.zeros(nt)
        nngb, iters = np.zeros(nt, np.int32), np.zeros(nt, np.int32)
        hs = _f64(h_start) if h_start is not None else None
        cp = _f64(cond_prev) if cond_prev is not None else None
        cs = np.zeros(nt + 1, np.int64) if cache else None
        args = [self.h, nt, _p(t, _u32), des_ngb, ngb_tol, _p(hs, _d), box, n_dims, _p(cp, _d), _p(h, _d),
                _p(rho, _d), nngb.ctypes.data, iters.ctypes.data]
        self.lib.L.ref_density(*args, _p(cs, _i64), None, 0)
        out = {"h": h, "rho": rho, "nngb": nngb, "iters": iters}
        if cache:
            flat = np.zeros(max(int(cs[-1]), 1), np.uint32)
            self.lib.L.ref_density(*args, _p(cs, _i64), _p(flat, _u32), len(flat))
            out["cache_start"], out["cache_flat"] = cs, flat[: cs[-1]]
        return out

    def vel_moments(self):
        nn = self.nnodes
        v = [np.zeros(nn) for _ in range(3)]
        vmax = np.zeros(nn, np.float32)
        self.lib.L.ref_tree_vel(self.h, _p(v[0], _d), _p(v[1], _d), _p(v[2], _d), _p(vmax, _f))
        return v, vmax

    def accel(self, targets, theta, G=1.0, aold=None):
        t = _targets(targets)
        nt = len(t)
        ax, ay, az = np.empty(nt), np.empty(nt), np.empty(nt)
        ao = _f64(aold) if aold is not None else None
        self.lib.L.ref_accel(self.h, nt, _p(t, _u32), theta, G, _p(ao, _d), _p(ax, _d),
                             _p(ay, _d), _p(az, _d))
        return ax, ay, az

    def potential(self, targets, theta, G=1.0, aold=None):
        t = _targets(targets)
        phi = np.empty(len(t))
        ao = _f64(aold) if aold is not None else None
        self.lib.L.ref_potential(self.h, len(t), _p(t, _u32), theta, G, _p(ao, _d), _p(phi, _d))
        return phi

    def accel_brute(self, targets, G=1.0):
        t = _targets(targets)
        nt = len(t)
        ax, ay, az = np.empty(nt), np.empty(nt), np.empty(nt)
        self.lib.L.ref_accel_brute(self.h, nt, _p(t, _u32), G, _p(ax, _d), _p(ay, _d), _p(az, _d))
        return ax, ay, az
