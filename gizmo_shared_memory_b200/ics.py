"""Seeded synthetic particle sets for the tree-gravity workloads.

The reference's real inputs (the BBB03 / M50 state files read by ``shmem/bench_treeforce.cc:21-32``)
are not available, so every workload is generated here from a stated seed with numpy's PCG64
generator.  Each generator returns a dict of FP64 numpy arrays ``x, y, z, m, soft`` (``soft`` is the
cubic-spline kernel extent h stored in ``shmem::Particles::soft``, shmem/tree.h:37).

* ``plummer``         — Plummer sphere, radii by the inverse cumulative mass profile truncated at
                         ``rmax`` (as ``shmem/test_tree.cc:96-107`` draws them), isotropic directions.
* ``galaxy``          — Hernquist halo (inverse of M(<r) = r^2/(r+a)^2, truncated) plus an
                         exponential disk (radius from 1-(1+x)e^{-x} = U, sech^2 vertical profile).
* ``soneira_peebles`` — hierarchical clustering in the unit cube (eta children per level, radius
                         shrinking by lambda per level), a uniform background fraction, folded into
                         the cube.
* ``plummer_batch``   — many independent Plummer spheres of uneven N (log-uniform), with per-system
                         scale radius and softening, for the batched multi-system walk.
* ``merger``          — two galaxies on a parabolic approach with a seeded relative rotation.
"""
from __future__ import annotations

import math

import numpy as np


def _isotropic(rng, n):
    ct = rng.uniform(-1.0, 1.0, n)
    st = np.sqrt(np.maximum(0.0, 1.0 - ct * ct))
    ph = rng.uniform(0.0, 2.0 * math.pi, n)
    return st * np.cos(ph), st * np.sin(ph), ct


def _pack(x, y, z, m, soft):
    return {
        "x": np.ascontiguousarray(x, np.float64),
        "y": np.ascontiguousarray(y, np.float64),
        "z": np.ascontiguousarray(z, np.float64),
        "m": np.ascontiguousarray(m, np.float64),
        "soft": np.ascontiguousarray(soft, np.float64),
    }


def plummer(n=65536, a=1.0, mass=1.0, rmax=20.0, soft=0.01, seed=42, center=(0.0, 0.0, 0.0)):
    """Plummer sphere of total mass ``mass`` truncated at ``rmax`` scale radii."""
    rng = np.random.default_rng(seed)
    q = rmax  # in units of a
    mtrunc = q ** 3 / (1.0 + q * q) ** 1.5
    X = rng.uniform(0.0, mtrunc, n)
    X = np.maximum(X, 1e-300)
    r = a / np.sqrt(X ** (-2.0 / 3.0) - 1.0)
    ux, uy, uz = _isotropic(rng, n)
    return _pack(center[0] + r * ux, center[1] + r * uy, center[2] + r * uz,
                 np.full(n, mass / n), np.full(n, soft))


def galaxy(n_halo=3_145_728, n_disk=1_048_576, m_halo=1.0, a_halo=1.0, r_trunc=30.0,
           m_disk=0.05, r_disk=0.1, z_disk=0.01, soft_halo=0.005, soft_disk=0.002, seed=2):
    """Hernquist halo plus exponential, sech^2 disk (the isolated-galaxy workload)."""
    from scipy.special import lambertw

    rng = np.random.default_rng(seed)
    q = r_trunc / a_halo
    mt = q * q / (1.0 + q) ** 2
    X = rng.uniform(0.0, mt, n_halo)
    s = np.sqrt(X)
    r = a_halo * s / (1.0 - s)
    ux, uy, uz = _isotropic(rng, n_halo)
    hx, hy, hz = r * ux, r * uy, r * uz
    U = rng.uniform(0.0, 1.0, n_disk)
    U = np.minimum(U, 1.0 - 1e-15)
    xr = -1.0 - np.real(lambertw((U - 1.0) / math.e, k=-1))
    R = r_disk * xr
    ph = rng.uniform(0.0, 2.0 * math.pi, n_disk)
    V = rng.uniform(-1.0 + 1e-15, 1.0 - 1e-15, n_disk)
    dz = z_disk * np.arctanh(V)
    x = np.concatenate([hx, R * np.cos(ph)])
    y = np.concatenate([hy, R * np.sin(ph)])
    z = np.concatenate([hz, dz])
    m = np.concatenate([np.full(n_halo, m_halo / n_halo), np.full(n_disk, m_disk / n_disk)])
    soft = np.concatenate([np.full(n_halo, soft_halo), np.full(n_disk, soft_disk)])
    return _pack(x, y, z, m, soft)


def soneira_peebles(levels=12, eta=4, lam=1.9, background=0.10, soft=1e-4, seed=3, radius=0.5):
    """Soneira-Peebles hierarchy in the unit cube: eta^levels points of equal mass."""
    rng = np.random.default_rng(seed)
    cx = np.array([0.5])
    cy = np.array([0.5])
    cz = np.array([0.5])
    R = radius
    for _ in range(levels):
        k = cx.size * eta
        # child centres uniform in the parent sphere of radius R; child radius R / lam
        rr = R * rng.uniform(0.0, 1.0, k) ** (1.0 / 3.0)
        ux, uy, uz = _isotropic(rng, k)
        cx = np.repeat(cx, eta) + rr * ux
        cy = np.repeat(cy, eta) + rr * uy
        cz = np.repeat(cz, eta) + rr * uz
        R = R / lam
    n = cx.size
    nb = int(round(background * n))
    pick = rng.choice(n, size=nb, replace=False)
    cx[pick] = rng.uniform(0.0, 1.0, nb)
    cy[pick] = rng.uniform(0.0, 1.0, nb)
    cz[pick] = rng.uniform(0.0, 1.0, nb)
    cx = np.mod(cx, 1.0)
    cy = np.mod(cy, 1.0)
    cz = np.mod(cz, 1.0)
    return _pack(cx, cy, cz, np.full(n, 1.0 / n), np.full(n, soft))


def plummer_batch(n_systems=256, n_min=1024, n_max=262144, n_total=1 << 24, a_min=0.5, a_max=2.0,
                  seed=4, spacing=None):
    """Independent Plummer spheres with log-uniform N and scale radius; returns (P, offsets, meta).

    N_i are drawn log-uniform in [n_min, n_max], then rescaled by one common factor so that
    sum N_i is about ``n_total`` (the raw mean gives only ~12M for the defaults).  Systems are laid
    out on a line ``spacing`` apart so a single tree could also hold them; the batched walk treats
    each system independently."""
    rng = np.random.default_rng(seed)
    raw = np.exp(rng.uniform(math.log(n_min), math.log(n_max), n_systems))
    scale = n_total / raw.sum()
    ns = np.maximum(1, np.round(raw * scale)).astype(np.int64)
    a = np.exp(rng.uniform(math.log(a_min), math.log(a_max), n_systems))
    if spacing is None:
        spacing = 200.0 * a_max
    parts = []
    for s in range(n_systems):
        parts.append(plummer(int(ns[s]), a=float(a[s]), soft=0.01 * float(a[s]),
                             seed=seed * 100003 + s, center=(s * spacing, 0.0, 0.0)))
    P = {k: np.concatenate([p[k] for p in parts]) for k in ("x", "y", "z", "m", "soft")}
    offsets = np.concatenate([[0], np.cumsum(ns)]).astype(np.int64)
    return P, offsets, {"n": ns, "a": a}


def _rotation(rng):
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([
        [1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
        [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
        [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)],
    ])


def merger(n_each=33_554_432, separation=20.0, seed=5):
    """Two isolated galaxies, each of n_each particles with particle masses halved, centres
    ``separation`` apart, the second rotated by a seeded random rotation."""
    n_disk = n_each // 4
    n_halo = n_each - n_disk
    g1 = galaxy(n_halo=n_halo, n_disk=n_disk, seed=seed)
    g2 = galaxy(n_halo=n_halo, n_disk=n_disk, seed=seed + 1)
    rng = np.random.default_rng(seed + 2)
    Rm = _rotation(rng)
    p2 = Rm @ np.vstack([g2["x"], g2["y"], g2["z"]])
    x = np.concatenate([g1["x"] - 0.5 * separation, p2[0] + 0.5 * separation])
    y = np.concatenate([g1["y"], p2[1]])
    z = np.concatenate([g1["z"], p2[2]])
    m = 0.5 * np.concatenate([g1["m"], g2["m"]])
    soft = np.concatenate([g1["soft"], g2["soft"]])
    return _pack(x, y, z, m, soft)


def config(name: str):
    """The named workloads with their stated sizes."""
    if name == "plummer_65k":
        return plummer()
    if name == "galaxy_4m":
        return galaxy()
    if name == "clustered_16m":
        return soneira_peebles()
    if name == "merger_67m":
        return merger()
    raise KeyError(name)


def write_state(path, P, vel):
    """The flat particle dump shmem/bench_treeforce.cc reads: N (u64), then x, y, z, m, h, vx, vy,
    vz as contiguous float64 arrays."""
    n = len(P["m"])
    with open(path, "wb") as fh:
        np.array([n], np.uint64).tofile(fh)
        for a in (P["x"], P["y"], P["z"], P["m"], P["soft"], vel[0], vel[1], vel[2]):
            np.ascontiguousarray(a, np.float64).tofile(fh)


def plummer_state(n=200000, seed=11, sigma=0.5):
    """A Plummer sphere with seeded Gaussian velocities: a synthetic stand-in for the engine state
    files bench_treeforce reads."""
    P = plummer(n=n, seed=seed, soft=0.01)
    rng = np.random.default_rng(seed + 1)
    vel = [rng.normal(0.0, sigma, n) for _ in range(3)]
    return P, vel
