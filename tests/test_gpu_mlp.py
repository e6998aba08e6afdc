"""Surrogate network kernels against the float64 CPU restatement."""
import numpy as np
import pytest

from tensum_b200 import mlp

import mlp_oracle as M  # noqa: E402

pytestmark = pytest.mark.gpu


def _net(din=3, dout=3, seed=1):
    net = mlp.MLP(din, dout, seed=seed)
    rng = np.random.default_rng(seed)
    theta = rng.normal(0.0, 0.25, net.np).astype(np.float32)
    net.params = theta
    return net, theta.astype(np.float64), rng


def test_gradient_matches_cpu_oracle():
    for din, dout in ((3, 3), (20, 3)):
        net, theta, rng = _net(din, dout)
        X = rng.normal(size=(200, din)).astype(np.float32)
        T = rng.normal(size=(200, dout)).astype(np.float32)
        loss, g = net.loss_grad(X, T)
        rl, rg = M.loss_grad(theta, X.astype(np.float64), T.astype(np.float64), din, dout)
        assert abs(loss - rl) <= 1e-5 * abs(rl)
        # FP32 kernels against float64: per parameter, relative to the largest gradient entry
        assert np.max(np.abs(g - rg)) <= 2e-5 * np.max(np.abs(rg))


def test_fp32_and_bf16_forward():
    net, theta, rng = _net(3, 3)
    X = rng.normal(size=(1000, 3)).astype(np.float32)
    ref, _ = M.forward(theta, X.astype(np.float64), 3, 3)
    y32 = net.raw_predict(X, precision=0)
    assert np.max(np.abs(y32 - ref)) <= 1e-5 * np.max(np.abs(ref))
    y16 = net.raw_predict(X, precision=1)       # BF16 tensor cores on the two 64x64 layers
    assert np.max(np.abs(y16 - ref)) <= 3e-2 * np.max(np.abs(ref))
    assert np.corrcoef(y16.ravel(), ref.ravel())[0, 1] > 0.999
    # ragged sizes: tiles of 16 samples with a partial last tile
    for n in (1, 15, 17, 333):
        assert np.allclose(net.raw_predict(X[:n], precision=1), y16[:n], rtol=0, atol=0)


def test_training_learns_and_is_reproducible():
    rng = np.random.default_rng(3)
    X = rng.uniform(-1, 1, size=(512, 3))
    Y = np.stack([np.sin(2 * X[:, 0]) + X[:, 1] ** 2, X[:, 0] * X[:, 2], np.cos(X[:, 1] + X[:, 2])], axis=1)
    losses = []
    params = []
    for _ in range(2):
        net = mlp.MLP(3, 3, seed=7)
        l = net.fit(X, Y, epochs=150, batch=64, lr=3e-3)
        losses.append(l)
        params.append(net.params)
    assert np.array_equal(params[0], params[1]) and np.array_equal(losses[0], losses[1])
    assert losses[0][-1] < 0.02 * losses[0][0]
    Xt = rng.uniform(-1, 1, size=(256, 3))
    Yt = np.stack([np.sin(2 * Xt[:, 0]) + Xt[:, 1] ** 2, Xt[:, 0] * Xt[:, 2], np.cos(Xt[:, 1] + Xt[:, 2])], axis=1)
    pred = net.predict(Xt, precision=1)
    assert np.sqrt(np.mean((pred - Yt) ** 2)) < 0.1 * Yt.std()
