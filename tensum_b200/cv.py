"""Multi-fidelity Monte Carlo with a surrogate control variate.

The expensive model is the solver (a QoI vector per sample); the cheap model
is the surrogate network g evaluated at the same random inputs.  With N paired
samples (Y_i, g(X_i)) and M further surrogate evaluations g(X'_j) at fresh
inputs, the control-variate estimator of E[Y] is

    mu_cv = mean(Y) - beta (mean(g(X)) - mean(g(X')))

with beta = Cov(Y, g) / Var(g) per QoI (the variance-minimising coefficient).
It is unbiased for any fixed beta because E[g(X)] = E[g(X')]; estimating beta
from the same N pairs adds an O(1/N) bias that the plain estimate bounds.  Its
variance is Var(Y - beta g)/N + beta^2 Var(g)/M against Var(Y)/N for plain MC.
Plain MC is both the fallback (used whenever the control variate does not
reduce the estimated variance) and the yardstick: every result reports the plain
estimate and the variance ratio next to the multi-fidelity one.  The surrogate
never replaces the solver.  The variance of Y is estimated the same way from
the second moment E[Y^2] with g^2 as its control.
"""
from __future__ import annotations

import numpy as np


def _cv(y, g, ge):
    N, M = y.shape[0], ge.shape[0]
    ym, gm, gem = y.mean(0), g.mean(0), ge.mean(0)
    vg = g.var(0, ddof=1)
    cov = ((y - ym) * (g - gm)).sum(0) / (N - 1)
    beta = np.where(vg > 0, cov / np.where(vg > 0, vg, 1.0), 0.0)
    mu = ym - beta * (gm - gem)
    var_cv = (y - beta * g).var(0, ddof=1) / N + beta ** 2 * ge.var(0, ddof=1) / M
    var_mc = y.var(0, ddof=1) / N
    return mu, var_cv, ym, var_mc, beta


def estimate(y, g, g_extra) -> dict:
    """Mean and variance of each QoI column by the control-variate estimator.

    y: (N, q) solver QoIs; g: (N, q) surrogate at the same inputs;
    g_extra: (M, q) surrogate at M fresh inputs.  Returns per QoI the estimates
    actually used ('mean', 'var', and their standard errors 'se_mean'), the
    plain Monte Carlo ones ('plain_mean', 'plain_var', 'plain_se_mean'), the
    control coefficients, the variance ratio of the mean estimators ('gain',
    > 1 when the surrogate helps) and 'used' (True where the control variate
    was used, False where plain MC took over)."""
    y = np.asarray(y, np.float64)
    g = np.asarray(g, np.float64)
    ge = np.asarray(g_extra, np.float64)
    if y.ndim == 1:
        y, g, ge = y[:, None], g[:, None], ge[:, None]
    mu, var_cv, ym, var_mc, beta = _cv(y, g, ge)
    m2, _, y2m, _, beta2 = _cv(y * y, g * g, ge * ge)
    gain = var_mc / np.maximum(var_cv, 1e-300)
    used = var_cv < var_mc
    mean = np.where(used, mu, ym)
    plain_var = y.var(0, ddof=1)
    var_est = np.where(used, m2 - mu * mu, plain_var)
    # the multi-fidelity variance estimate uses the (N-1)/N sample correction of the plain one
    var_est = np.where(used, var_est * y.shape[0] / (y.shape[0] - 1), var_est)
    return dict(mean=mean, var=var_est, se_mean=np.sqrt(np.where(used, var_cv, var_mc)),
                plain_mean=ym, plain_var=plain_var, plain_se_mean=np.sqrt(var_mc),
                beta=beta, beta_second=beta2, gain=gain, used=used, n=y.shape[0], m=ge.shape[0])


def samples_for_rse(y, g=None, rse: float = 0.01) -> np.ndarray:
    """Expensive samples needed for a relative standard error `rse` of the mean:
    plain MC when g is None, else the control-variate estimator with an
    unlimited surrogate budget (the Var(g)/M term vanishes)."""
    y = np.asarray(y, np.float64)
    if y.ndim == 1:
        y = y[:, None]
    mu = np.abs(y.mean(0))
    if g is None:
        v = y.var(0, ddof=1)
    else:
        g = np.asarray(g, np.float64)
        if g.ndim == 1:
            g = g[:, None]
        _, _, _, _, beta = _cv(y, g, g)
        v = (y - beta * g).var(0, ddof=1)
    return np.ceil(v / (rse * mu) ** 2)


def samples_for_rse_var(y, g=None, rse: float = 0.01) -> np.ndarray:
    """Expensive samples needed for a relative standard error `rse` of the
    variance estimate: Var((Y - E Y)^2) / (rse Var Y)^2 for plain MC; with the
    surrogate, the squared deviations get (g - E g)^2 as their control
    (unlimited surrogate budget), Var(Z - beta G) / (rse Var Y)^2."""
    y = np.asarray(y, np.float64)
    if y.ndim == 1:
        y = y[:, None]
    z = (y - y.mean(0)) ** 2
    target = (rse * y.var(0, ddof=1)) ** 2
    if g is None:
        return np.ceil(z.var(0, ddof=1) / target)
    g = np.asarray(g, np.float64)
    if g.ndim == 1:
        g = g[:, None]
    gz = (g - g.mean(0)) ** 2
    _, _, _, _, beta = _cv(z, gz, gz)
    return np.ceil((z - beta * gz).var(0, ddof=1) / target)


def rse_now(y, g=None, g_extra=None) -> tuple[np.ndarray, np.ndarray]:
    """Current relative standard errors of the mean and of the variance estimate
    of each QoI column, from the N samples in hand (the stopping rule of a
    sequential Monte Carlo run).

    Plain MC (g None): se(mean) = sqrt(Var Y / N), se(var) = sqrt(Var Z / N)
    with Z = (Y - mean Y)^2.  With the surrogate (g at the same inputs, g_extra
    at M fresh ones) the mean gets the control-variate standard error of
    `estimate` and Z gets (g - mean g_extra)^2 as its control, each with the
    surrogate's own sampling term beta^2 Var / M; where the control does not
    reduce the error, the plain one is used, as `estimate` falls back."""
    y = np.asarray(y, np.float64)
    if y.ndim == 1:
        y = y[:, None]
    N = y.shape[0]
    mu, var = y.mean(0), y.var(0, ddof=1)
    z = (y - mu) ** 2
    se_m, se_v = np.sqrt(var / N), np.sqrt(z.var(0, ddof=1) / N)
    if g is not None:
        g = np.asarray(g, np.float64).reshape(y.shape)
        ge = np.asarray(g_extra, np.float64)
        ge = ge.reshape(ge.shape[0], -1)
        _, var_cv, _, _, _ = _cv(y, g, ge)
        gem = ge.mean(0)
        gz, gze = (g - gem) ** 2, (ge - gem) ** 2
        _, var_cvz, _, _, _ = _cv(z, gz, gze)
        se_m = np.minimum(se_m, np.sqrt(var_cv))
        se_v = np.minimum(se_v, np.sqrt(var_cvz))
    return se_m / np.abs(mu), se_v / var
