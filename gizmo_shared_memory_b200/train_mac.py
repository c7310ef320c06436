"""Train the per-node learned opening criterion (GT_MAC_NODE) on the GPU and write the model.

Training data come from the plain walk on the two training workloads -- the 65,536-particle
Plummer sphere and the 4M isolated galaxy -- exactly as the learned criterion is specified: for
sampled (window of 32 targets, node) pairs of a walk with the relative criterion, the exact error
of accepting the node (its monopole against the sum over its particles) and the geometry
features (gt_mac_sample).  The network is trained by the library's own kernels (gt_mac_train:
pinball loss at quantile tau, Adam) on two node-only features -- the node's second mass moment
q2 / (M L^2) and its centre-of-mass offset delta / L -- so the walk can evaluate it once per node.
The particle count, the third node-only feature, is left out: near the acceptance threshold it
carries no signal in the training workloads, and models that read it did worse out of
distribution (on the 16M clustered box, 0.971x the plain criterion's interactions at equal p99
with it, 1.025x without it).

    python -m gizmo_shared_memory_b200.train_mac [--out PATH] [--tau 0.5] [--epochs 20]

The default output is mac_node_model.npy beside this file: 1393 float32 (include/gt.h model
layout), plus a JSON sidecar with the training settings and the median prediction (the kappa
scale of the model).
"""
from __future__ import annotations

import argparse
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_OUT = os.path.join(HERE, "mac_node_model.npy")
# node features the network reads: 1 = log q2 / (M L^2), 2 = log delta / L (gt_mac.cuh)
FEATURE_MASK = (1 << 1) | (1 << 2)


def training_samples(ctx, alpha=0.0025, galaxy_stride=16):
    import torch

    from . import _gt as gtm
    from . import ics

    feats, labs = [], []
    for P, stride in ((ics.plummer(n=65536, seed=42), 1), (ics.galaxy(seed=2), galaxy_stride)):
        dev = {k: torch.as_tensor(v, device="cuda") for k, v in P.items()}
        T = ctx.build(dev)
        nl = T.info()["n_live"]
        out = tuple(torch.empty(nl, dtype=torch.float64, device="cuda") for _ in range(3))
        W = dict(group_mode=gtm.GT_GROUP_BATCH, batch=32)
        ctx.accel_grouped(T, None, theta=0.7, outs=out + (None,), **W)
        aold = ctx.form_aold(*out, 0.0005)
        ctx.accel_grouped(T, None, aold=aold, outs=out + (None,), **W)  # an accurate |a|
        amag = torch.sqrt(out[0] ** 2 + out[1] ** 2 + out[2] ** 2)
        f, lab, _, _ = ctx.mac_sample(T, amag, alpha=alpha, window=32, stride=stride, rho_lo=0.01,
                                      rho_hi=100.0, capacity=1 << 21)
        feats.append(f)
        labs.append(lab)
    X = np.concatenate(feats)
    Y = np.concatenate(labs)
    ok = np.isfinite(X).all(1) & np.isfinite(Y)
    return X[ok], Y[ok]


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--out", default=DEFAULT_OUT)
    ap.add_argument("--tau", type=float, default=0.5)
    ap.add_argument("--epochs", type=int, default=20)
    ap.add_argument("--seed", type=int, default=1)
    args = ap.parse_args(argv)
    sys.path.insert(0, os.path.dirname(HERE))
    import gizmo_shared_memory_b200 as g

    ctx = g.Context(0, torch_stream=True)
    X, Y = training_samples(ctx)
    mask = FEATURE_MASK
    model, loss = ctx.mac_train(X, Y, epochs=args.epochs, batch=4096, lr=2e-3, tau=args.tau, seed=args.seed,
                                feature_mask=mask)
    pred = ctx.mac_predict(model, X)
    np.save(args.out, model.astype(np.float32))
    meta = {"tau": args.tau, "epochs": args.epochs, "seed": args.seed, "samples": int(len(Y)), "loss": loss,
            "median_prediction": float(np.median(pred)),
            "training": "plummer N=65536 seed 42 (every window) + galaxy 4M seed 2 (every 16th window), "
                        "alpha 0.0025, windows of 32, rho in [0.01, 100]",
            "feature_mask": int(mask)}
    with open(os.path.splitext(args.out)[0] + ".json", "w") as fh:
        json.dump(meta, fh, indent=1)
    print(json.dumps(meta))


if __name__ == "__main__":
    main()
