"""The cylinder control-variate pipeline end to end on a small O-mesh.

Batched FP32 solves and FP64 solves (concurrent handles) of the same
uncertain inputs give the same QoIs within FP32 tolerances; a surrogate
trained on part of the batch serves as control variate for the rest.
"""
import numpy as np
import pytest

from tensum_b200 import cases, cv, cylinder, mlp, preproc

pytestmark = pytest.mark.gpu


def test_batched_fp32_and_fp64_qois_agree_and_the_surrogate_helps():
    m = cases.cylinder_mesh(16, 32, 2)
    g = preproc.preprocess(m)
    X = cylinder.draw_inputs(128, 5)
    T, n_out, t0 = 0.1, 10, 0.05
    rb = cylinder.run_batched(g, m.coords, X, T, n_out, t0, tune=False)
    assert rb["bad"] == 0
    r64 = cylinder.run_fp64(g, m.coords, X[:6], T, n_out, t0, streams=3)
    y, y64 = rb["y"], r64["y"]
    assert np.all(np.isfinite(y)) and np.all(np.isfinite(y64))
    np.testing.assert_allclose(rb["times"], np.linspace(0.0, T, n_out + 1))
    # drag and its viscous share: FP32 members within 1e-4 relative; the lift
    # fluctuation is a small difference of large forces: within 1e-3 of the drag
    assert np.max(np.abs(y[:6, 0] - y64[:, 0]) / np.abs(y64[:, 0])) < 1e-4
    assert np.max(np.abs(y[:6, 2] - y64[:, 2]) / np.abs(y64[:, 2])) < 1e-4
    assert np.max(np.abs(y[:6, 1] - y64[:, 1])) < 1e-3 * np.min(np.abs(y64[:, 0]))
    # the force history itself
    f32, f64 = rb["forces"][:6], r64["forces"]
    assert np.max(np.abs(f32 - f64)) <= 1e-4 * np.max(np.abs(f64))
    net = mlp.MLP(3, 3, seed=0)
    net.fit(X[:64], y[:64], epochs=300, batch=32, lr=3e-3)
    r = cv.estimate(y[64:], net.predict(X[64:]), net.predict(cylinder.draw_inputs(1 << 14, 9)))
    assert r["gain"][0] > 4.0, r["gain"]
