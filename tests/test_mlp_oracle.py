"""The CPU restatement of the surrogate network against finite differences."""
import numpy as np

import mlp_oracle as M  # noqa: E402  (oracle/ is on sys.path for the tests)


def test_oracle_gradient_matches_central_differences():
    rng = np.random.default_rng(0)
    din, dout = 3, 3
    n_par = M.H * din + M.H + 2 * (M.H * M.H + M.H) + dout * M.H + dout
    theta = rng.normal(0.0, 0.3, n_par)
    X = rng.normal(size=(17, din))
    T = rng.normal(size=(17, dout))
    _, g = M.loss_grad(theta, X, T, din, dout)
    idx = rng.choice(n_par, 60, replace=False)
    h = 1e-6
    for p in idx:
        e = np.zeros(n_par)
        e[p] = h
        num = (M.loss_grad(theta + e, X, T, din, dout)[0] - M.loss_grad(theta - e, X, T, din, dout)[0]) / (2 * h)
        assert abs(num - g[p]) <= 1e-7 + 1e-5 * abs(num), p
