"""CPU restatement of the surrogate network for gradient checks (test infrastructure).

Forward and backward of din -> 64 -> 64 -> 64 -> dout with exact GELU
(0.5 x (1 + erf(x / sqrt 2))) and mean squared error, in float64 with numpy,
over the parameter vector layout of tg_mlp (W1[64][din] b1 W2 b2 W3 b3
W4[dout][64] b4).  The network has no counterpart in the reference; this file
is checked against central finite differences in tests/test_mlp_oracle.py.
"""
from __future__ import annotations

import numpy as np
from scipy.special import erf

H = 64


def unpack(theta, din, dout):
    theta = np.asarray(theta, np.float64)
    o = 0
    out = []
    for shape in [(H, din), (H,), (H, H), (H,), (H, H), (H,), (dout, H), (dout,)]:
        n = int(np.prod(shape))
        out.append(theta[o:o + n].reshape(shape))
        o += n
    assert o == theta.size
    return out


def gelu(x):
    return 0.5 * x * (1.0 + erf(x / np.sqrt(2.0)))


def gelu_d(x):
    return 0.5 * (1.0 + erf(x / np.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / np.sqrt(2.0 * np.pi)


def forward(theta, X, din, dout):
    W1, b1, W2, b2, W3, b3, W4, b4 = unpack(theta, din, dout)
    z1 = X @ W1.T + b1
    a1 = gelu(z1)
    z2 = a1 @ W2.T + b2
    a2 = gelu(z2)
    z3 = a2 @ W3.T + b3
    a3 = gelu(z3)
    y = a3 @ W4.T + b4
    return y, (z1, a1, z2, a2, z3, a3)


def loss_grad(theta, X, T, din, dout):
    X = np.asarray(X, np.float64)
    T = np.asarray(T, np.float64)
    W1, b1, W2, b2, W3, b3, W4, b4 = unpack(theta, din, dout)
    y, (z1, a1, z2, a2, z3, a3) = forward(theta, X, din, dout)
    n = X.shape[0]
    loss = np.sum((y - T) ** 2) / (n * dout)
    d4 = 2.0 * (y - T) / (n * dout)
    d3 = (d4 @ W4) * gelu_d(z3)
    d2 = (d3 @ W3) * gelu_d(z2)
    d1 = (d2 @ W2) * gelu_d(z1)
    g = [d1.T @ X, d1.sum(0), d2.T @ a1, d2.sum(0), d3.T @ a2, d3.sum(0), d4.T @ a3, d4.sum(0)]
    return loss, np.concatenate([x.ravel() for x in g])
