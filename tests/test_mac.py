"""Learned opening criterion: the numpy oracle of the network (oracle/mlp.py) checked by finite
differences (CPU), and the library's training and inference kernels checked against it (GPU)."""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import mlp  # noqa: E402


def random_model(rng):
    m = np.zeros(mlp.MODEL)
    m[:8] = rng.normal(size=8)
    m[8:16] = rng.uniform(0.5, 2.0, 8)
    m[16:] = rng.normal(scale=0.3, size=mlp.PARAMS)
    return m


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    m = random_model(rng)
    X = rng.normal(size=(64, 8))
    Y = rng.normal(size=64)
    loss, g = mlp.loss_and_grad(m, X, Y, 0.9)
    assert g.shape == (mlp.PARAMS,)
    for idx in rng.choice(mlp.PARAMS, 60, replace=False):
        fd = mlp.finite_difference(m, X, Y, 0.9, idx)
        assert fd == pytest.approx(g[idx], rel=1e-4, abs=1e-8)


@pytest.mark.gpu
def test_gpu_gradient_and_prediction_match_oracle(gpu_ctx):
    rng = np.random.default_rng(1)
    m = random_model(rng).astype(np.float32)
    X = rng.normal(size=(3000, 8)).astype(np.float32)
    Y = rng.normal(size=3000).astype(np.float32)
    g, loss = gpu_ctx.mac_gradient(m, X, Y, tau=0.9)
    rloss, rg = mlp.loss_and_grad(m.astype(np.float64), X.astype(np.float64), Y.astype(np.float64), 0.9)
    assert loss == pytest.approx(rloss, rel=1e-5)
    assert np.abs(g - rg).max() <= 1e-4 * np.abs(rg).max()
    p = gpu_ctx.mac_predict(m, X)
    rp, _ = mlp.forward(m.astype(np.float64), X.astype(np.float64))
    assert np.abs(p - rp).max() <= 1e-4 * (1 + np.abs(rp).max())


@pytest.mark.gpu
def test_gpu_training_fits_a_smooth_function(gpu_ctx):
    rng = np.random.default_rng(2)
    X = rng.uniform(-2, 2, size=(40000, 8)).astype(np.float32)
    Y = (np.sin(X[:, 0]) + 0.5 * X[:, 1] * X[:, 2] - 0.3 * X[:, 3]).astype(np.float32)
    Y += 0.05 * rng.normal(size=len(Y)).astype(np.float32)
    model, loss = gpu_ctx.mac_train(X, Y, epochs=25, batch=2048, lr=3e-3, tau=0.5)
    pred = gpu_ctx.mac_predict(model, X)
    base = np.abs(Y - np.median(Y)).mean() * 0.5
    assert loss < 0.25 * base  # median regression: pinball(0.5) = |r|/2
    assert np.mean(np.abs(pred - Y)) < 0.2
