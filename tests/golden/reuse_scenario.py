"""The tree-reuse scenario shared by tests/golden/make_golden.py and the reuse tests: a seeded
sequence of incremental-moment events (shmem/tree.cc:211-329) on the 4096-particle Plummer sphere
of the fixtures, by particle index (each tree maps particles to its own leaves), then the
particles' positions a time tau later."""
import numpy as np

TAU = 0.05
# event kinds as include/gt.h numbers them
KICK, SHIFT, VMAX, SOFT, MASS, PAD = range(6)


def events(P, vel, seed=5):
    """[(kind, particles, arrays, tau)], in the order they are applied."""
    rng = np.random.default_rng(seed)
    live = np.nonzero(P["m"] > 0)[0]
    V = np.stack(vel, 1)
    X = np.stack([P["x"], P["y"], P["z"]], 1)
    out = []
    k = rng.choice(live, 1000, replace=False)
    out.append((KICK, k, {"a": P["m"][k, None] * rng.normal(0.0, 0.05, (len(k), 3))}, 0.02))
    s = rng.choice(live, 500, replace=False)
    out.append((VMAX, s, {"f": (np.linalg.norm(V[s], axis=1) * 1.5 + 0.1).astype(np.float32)}, 0.0))
    sh = rng.choice(live, 200, replace=False)
    out.append((SHIFT, sh, {"a": P["m"][sh], "x": rng.normal(0.0, 1e-3, (len(sh), 3))}, 0.0))
    me = rng.choice(live, 20, replace=False)
    dm = P["m"][me] * np.where(rng.uniform(size=len(me)) < 0.5, -0.5, 0.5)
    out.append((MASS, me, {"a": dm, "x": X[me] + V[me] * 0.03, "v": V[me]}, 0.03))
    pd = rng.choice(live, 50, replace=False)
    out.append((PAD, pd, {"a": rng.uniform(0.0, 1e-3, len(pd))}, 0.0))
    so = rng.choice(live, 30, replace=False)
    out.append((SOFT, so, {"a": P["soft"][so] * 1.5}, 0.0))
    return out


def positions_after(P, vel, evs, tau=TAU):
    """Ballistic positions at tau, plus the non-ballistic shifts of the SHIFT events."""
    x = P["x"] + vel[0] * tau
    y = P["y"] + vel[1] * tau
    z = P["z"] + vel[2] * tau
    for kind, parts, arr, _ in evs:
        if kind == SHIFT:
            x[parts] += arr["x"][:, 0]
            y[parts] += arr["x"][:, 1]
            z[parts] += arr["x"][:, 2]
    return x, y, z
