"""The trained surrogate as a control variate for Kelvin-Helmholtz ensembles.

Solver samples come from the batched FP32 engine; the surrogate (20 random
numbers -> 3 integrals) is trained on solver data by the network kernels and
evaluated in BF16.  The test shows what the network gains: the variance ratio
against plain Monte Carlo on the same expensive samples, with the estimate
consistent with a large plain ensemble.
"""
import numpy as np
import pytest

from tensum_b200 import abi, batch, cases, cv, mlp, preproc

pytestmark = pytest.mark.gpu


def _qoi(P, seeds):
    b = batch.Batch([(P, len(seeds))])
    rows = np.stack([cases.kh_rnd_row(int(s)) for s in seeds])
    b.set_kh(0, rows)
    b.advance(1)
    return rows, b.integrals(0)


def test_surrogate_control_variate_reduces_variance_without_bias():
    m = cases.kh_mesh(33, 0)
    cfg = dict(flux="kepes_tecno_rusanov", reconstruct="minmod", boundary={t: ("periodic", {}) for t in (1, 2, 3, 4)},
               final_time=0.1, time_stamps=1, cfl=0.8)
    P = abi.Problem(preproc.preprocess(m), cfg)
    x_tr, y_tr = _qoi(P, range(0, 1024))
    x_ev, y_ev = _qoi(P, range(10000, 10256))
    _, y_ref = _qoi(P, range(20000, 24096))
    net = mlp.MLP(20, 3, seed=5)
    net.fit(x_tr, y_tr, epochs=300, batch=128, lr=2e-3)
    x_ex = np.stack([cases.kh_rnd_row(s) for s in range(100000, 165536)])
    r = cv.estimate(y_ev, net.predict(x_ev), net.predict(x_ex))
    ref_mean = y_ref.mean(0)
    ref_se = y_ref.std(0, ddof=1) / np.sqrt(len(y_ref))
    # the vertical kinetic energy depends smoothly on the amplitudes: a large
    # gain; the weakly varying horizontal energy and entropy gain less, and the
    # estimator never does worse than plain MC (it falls back to it)
    assert r["gain"][0] > 4.0 and r["used"][0], r["gain"]
    assert np.all(r["gain"][1:] > 1.0), r["gain"]
    z = np.abs(r["mean"] - ref_mean) / np.sqrt(r["se_mean"] ** 2 + ref_se ** 2)
    assert np.all(z < 4.5), z
    # variance of the QoIs against the large plain ensemble
    assert abs(r["var"][0] / y_ref.var(0, ddof=1)[0] - 1.0) < 0.35
