"""ORACLE — test infrastructure only.

CPU restatement (numpy, per-event loops) of the reference's tree reuse: the incremental node
moments and the refreshed walk nodes of shmem/tree.cc:211-329 and tree.h:286-341 (GIZMO's
force_update_tree / force_kick_node / force_drift_node).  It works on the node arrays of an oracle
tree (oracle.RestatementTree, whose numbering is the reference's), applies events one at a time
in the reference's order and semantics, and writes the refreshed walk nodes back into the oracle
tree so its walk can run on the reused tree.  Pinned against the reference's own results in
tests/golden/golden.npz (``reuse_*``).
"""
from __future__ import annotations

import numpy as np


def _up_float(h):
    """h rounded up to float32 (tree.cc:288-291, h_as_bound)."""
    f = np.float32(h)
    return np.nextafter(f, np.float32(1e30)) if float(f) < h else f


def _min_image(s, box):
    """shmem/vec.h:25-31."""
    if box > 0:
        if s > 0.5 * box:
            s -= box
        elif s < -0.5 * box:
            s += box
    return s


class Reuse:
    def __init__(self, nodes, vcom=None, vmax=None, nodelta=False):
        """nodes: an oracle tree's nodes() dict; vcom: 3 arrays (node centre-of-mass velocity) or
        None; vmax: float32 node speed bounds (zeros without velocities)."""
        nn = len(nodes["mass"])
        self.parent = np.asarray(nodes["parent"])
        self.m0 = np.array(nodes["mass"], np.float64)
        self.c0 = np.stack([nodes["cx"], nodes["cy"], nodes["cz"]], 1).astype(np.float64)
        self.size = np.asarray(nodes["size"], np.float64)
        self.delta = np.asarray(nodes["delta"], np.float64)
        self.w_soft = np.array(nodes["w_soft"], np.float32)
        self.soft = np.array(nodes["soft"], np.float64)
        self.vcom = None if vcom is None else np.stack(vcom, 1).astype(np.float64)
        self.vmax = np.zeros(nn, np.float32) if vmax is None else np.array(vmax, np.float32)
        self.dp = np.zeros((nn, 3))
        self.dq = np.zeros((nn, 3))
        self.dmass = np.zeros(nn)
        self.xpad = np.zeros(nn, np.float32)
        self.nodelta = nodelta

    def _chain(self, leaf):
        no = int(leaf)
        while no >= 0:
            yield no
            no = int(self.parent[no])

    def node_mass(self, no):  # tree.h:327
        return self.m0[no] + self.dmass[no]

    def node_com(self, no, tau):  # tree.cc:228-236
        M = self.node_mass(no)
        if self.vcom is None or M <= 0:
            return self.c0[no].copy()
        m0 = self.m0[no]
        return (m0 * self.c0[no] + (m0 * self.vcom[no] + self.dp[no]) * tau - self.dq[no]) / M

    def node_vel(self, no):  # tree.h:333-341
        M = self.node_mass(no)
        if self.vcom is None or M <= 0:
            return None if self.vcom is None else self.vcom[no].copy()
        return (self.m0[no] * self.vcom[no] + self.dp[no]) / M

    def kick(self, leaf, dp, tau):  # tree.cc:211-226
        if self.vcom is None:
            return
        for no in self._chain(leaf):
            self.dp[no] += dp
            self.dq[no] += dp * tau

    def shift(self, leaf, m, dx):  # tree.cc:248-253
        if self.vcom is None or leaf < 0:
            return
        for no in self._chain(leaf):
            self.dq[no] -= m * np.asarray(dx)

    def raise_vmax(self, leaf, speed):  # tree.cc:276-284
        s = np.float32(speed)
        for no in self._chain(leaf):
            if self.vmax[no] >= s:
                return
            self.vmax[no] = max(self.vmax[no], s)

    def raise_soft(self, leaf, soft):  # tree.cc:310-319
        if leaf < 0:
            return
        sf = _up_float(soft)
        for no in self._chain(leaf):
            if self.w_soft[no] >= sf:
                return
            self.w_soft[no] = max(self.w_soft[no], sf)
            self.soft[no] = max(self.soft[no], soft)

    def mass_event(self, leaf, dm, x, v, tau, box=0.0):  # tree.cc:229-246
        if self.vcom is None or leaf < 0 or dm == 0.0:
            return
        for no in self._chain(leaf):
            c = self.node_com(no, tau)
            xr = np.array([c[k] + _min_image(x[k] - c[k], box) for k in range(3)])
            self.dmass[no] += dm
            self.dp[no] += dm * np.asarray(v)
            self.dq[no] -= dm * (xr - np.asarray(v) * tau)

    def raise_pad(self, leaf, d):  # tree.cc:322-329
        if leaf < 0 or not d > 0:
            return
        pad = _up_float(float(self.xpad[leaf]) + d)
        for no in self._chain(leaf):
            if self.xpad[no] >= pad:
                return
            self.xpad[no] = pad

    def events(self, kind, leaf, a=None, x=None, v=None, f=None, tau=0.0, box=0.0):
        """Events of one kind in order; kinds as include/gt.h numbers them."""
        for e, lf in enumerate(np.asarray(leaf)):
            lf = int(lf)
            if kind == 0:
                self.kick(lf, np.asarray(a[e], np.float64), tau)
            elif kind == 1:
                self.shift(lf, float(a[e]), x[e])
            elif kind == 2:
                self.raise_vmax(lf, f[e])
            elif kind == 3:
                self.raise_soft(lf, float(a[e]))
            elif kind == 4:
                self.mass_event(lf, float(a[e]), x[e], v[e], tau, box)
            elif kind == 5:
                self.raise_pad(lf, float(a[e]))

    def refresh(self, tau):  # tree.cc:256-274
        nn = len(self.m0)
        com = np.array([self.node_com(i, tau) for i in range(nn)])
        mass = self.m0 + self.dmass
        grow = 2.0 * (self.vmax.astype(np.float64) * tau + self.xpad.astype(np.float64))
        w_s = self.size + (0.0 if self.nodelta else self.delta) + grow
        w_len = (self.size + grow).astype(np.float32)
        vel = None
        if self.vcom is not None:
            vel = np.array([self.node_vel(i) for i in range(nn)])
        return {"com": com, "mass": mass, "w_s": w_s, "w_len": w_len, "w_soft": self.w_soft.copy(),
                "vmax": self.vmax.copy(), "xpad": self.xpad.copy(), "vel": vel}
