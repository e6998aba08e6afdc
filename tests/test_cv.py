"""Control-variate estimator on synthetic correlated data with known answers."""
import numpy as np

from tensum_b200 import cv


def _draw(rng, n, rho=0.98):
    x = rng.normal(size=(n, 2))
    y = np.stack([3.0 + x[:, 0], 1.0 + 0.5 * x[:, 1] ** 2], axis=1)
    g = np.stack([3.0 + rho * x[:, 0] + np.sqrt(1 - rho ** 2) * rng.normal(size=n) + 0.2,   # biased surrogate
                  1.0 + 0.5 * x[:, 1] ** 2 + 0.05 * rng.normal(size=n)], axis=1)
    return x, y, g


def test_unbiased_and_variance_reduced():
    rng = np.random.default_rng(0)
    true_mean = np.array([3.0, 1.5])
    errs_cv, errs_mc = [], []
    for rep in range(300):
        _, y, g = _draw(rng, 64)
        _, _, ge = _draw(rng, 20000)
        r = cv.estimate(y, g, ge)
        assert np.all(r["used"]) and np.all(r["gain"] > 5)
        errs_cv.append(r["mean"] - true_mean)
        errs_mc.append(r["plain_mean"] - true_mean)
    errs_cv, errs_mc = np.array(errs_cv), np.array(errs_mc)
    # a constant surrogate bias (0.2) does not bias the estimator
    assert np.all(np.abs(errs_cv.mean(0)) < 3 * errs_cv.std(0) / np.sqrt(len(errs_cv)) + 1e-3)
    assert np.all(errs_cv.var(0) < errs_mc.var(0) / 5)


def test_plain_mc_takes_over_for_a_useless_surrogate():
    rng = np.random.default_rng(1)
    y = rng.normal(size=(200, 1)) + 2.0
    g = rng.normal(size=(200, 1))              # independent of y
    ge = rng.normal(size=(1000, 1))
    r = cv.estimate(y, g, ge)
    if not r["used"][0]:
        assert r["mean"][0] == r["plain_mean"][0]
    assert r["gain"][0] < 1.2


def test_variance_estimate_and_sample_counts():
    rng = np.random.default_rng(2)
    _, y, g = _draw(rng, 4000)
    _, _, ge = _draw(rng, 100000)
    r = cv.estimate(y, g, ge)
    assert np.allclose(r["var"], [1.0, 0.5], rtol=0.1)
    n_mc = cv.samples_for_rse(y, None, 0.01)
    n_cv = cv.samples_for_rse(y, g, 0.01)
    assert np.all(n_cv < n_mc)


def test_variance_sample_counts():
    """Gaussian Y: Var((Y - mu)^2) = 2 sigma^4, so plain MC needs 2 / rse^2 samples
    for the variance; a close surrogate needs far fewer."""
    rng = np.random.default_rng(3)
    x = rng.normal(size=200000)
    y = 2.0 + 0.3 * x
    n = cv.samples_for_rse_var(y, None, 0.01)[0]
    assert abs(n / 20000.0 - 1.0) < 0.03
    g = 2.0 + 0.3 * x + 0.01 * rng.normal(size=x.size)
    assert cv.samples_for_rse_var(y, g, 0.01)[0] < n / 50
