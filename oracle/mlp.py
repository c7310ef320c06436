"""ORACLE — test infrastructure only.

numpy reference of the learned opening criterion's network (8 -> 32 -> 32 -> 1, ReLU, FP64
arithmetic) and of its training loss: the pinball (quantile) loss at quantile tau, averaged over
the batch, and its gradient with respect to the trainable parameters.  The layout is the one of
include/gt.h: model = [mean[8], 1/std[8], W1[32][8], b1[32], W2[32][32], b2[32], W3[32], b3].
Only the tests import it, to check the library's training and inference kernels.
"""
import numpy as np

NIN, NH = 8, 32
NORM = 2 * NIN
SIZES = [("W1", (NH, NIN)), ("b1", (NH,)), ("W2", (NH, NH)), ("b2", (NH,)), ("W3", (NH,)), ("b3", (1,))]
PARAMS = sum(int(np.prod(s)) for _, s in SIZES)
MODEL = NORM + PARAMS


def unpack(model):
    model = np.asarray(model, np.float64)
    out = {"mean": model[:NIN], "inv_sd": model[NIN:NORM]}
    o = NORM
    for name, shape in SIZES:
        n = int(np.prod(shape))
        out[name] = model[o:o + n].reshape(shape)
        o += n
    return out


def forward(model, X):
    p = unpack(model)
    xn = (np.asarray(X, np.float64) - p["mean"]) * p["inv_sd"]
    z1 = xn @ p["W1"].T + p["b1"]
    h1 = np.maximum(z1, 0.0)
    z2 = h1 @ p["W2"].T + p["b2"]
    h2 = np.maximum(z2, 0.0)
    y = h2 @ p["W3"] + p["b3"][0]
    return y, (xn, h1, h2)


def loss_and_grad(model, X, Y, tau):
    """Mean pinball loss and its gradient (flat, trainable-parameter layout)."""
    p = unpack(model)
    y, (xn, h1, h2) = forward(model, X)
    r = np.asarray(Y, np.float64) - y
    B = len(r)
    loss = np.where(r >= 0, tau * r, (tau - 1.0) * r).mean()
    dy = np.where(r >= 0, -tau, 1.0 - tau) / B
    gW3 = h2.T @ dy
    gb3 = np.array([dy.sum()])
    d2 = (dy[:, None] * p["W3"][None, :]) * (h2 > 0)
    gW2 = d2.T @ h1
    gb2 = d2.sum(0)
    d1 = (d2 @ p["W2"]) * (h1 > 0)
    gW1 = d1.T @ xn
    gb1 = d1.sum(0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3, gb3])
    return loss, g


def finite_difference(model, X, Y, tau, idx, eps=1e-6):
    """Central difference of the loss in trainable parameter idx (for checking loss_and_grad)."""
    m1 = np.array(model, np.float64)
    m2 = np.array(model, np.float64)
    m1[NORM + idx] += eps
    m2[NORM + idx] -= eps
    return (loss_and_grad(m1, X, Y, tau)[0] - loss_and_grad(m2, X, Y, tau)[0]) / (2 * eps)
