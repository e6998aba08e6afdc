"""Cylinder QoI post-processing on synthetic force histories."""
import numpy as np

from tensum_b200 import qoi


def test_force_coefficients_rotate_into_the_free_stream():
    # a force along the free stream at 30 degrees is pure drag
    f = np.array([[np.cos(np.pi / 6), np.sin(np.pi / 6), 0.0, 0.0],
                  [0.0, 0.0, -np.sin(np.pi / 6), np.cos(np.pi / 6)]])
    cd, cl = qoi.force_coefficients(f, 0.2, 30.0)
    q = 0.5 * 0.2 ** 2
    assert np.allclose(cd, [1 / q, 0.0], atol=1e-12)
    assert np.allclose(cl, [0.0, 1 / q], atol=1e-12)


def test_cylinder_qoi_of_a_sinusoidal_lift():
    mach, st = 0.2, 0.165
    t = np.linspace(0.0, 200.0, 20001)
    cl = 0.3 * np.sin(2 * np.pi * st * mach * t) + 0.05
    cd = 1.35 + 0.01 * np.cos(4 * np.pi * st * mach * t)
    m = qoi.cylinder_qoi(t, cd, cl, mach, t_start=50.0)
    assert abs(m[0] - 1.35) < 2e-3
    assert abs(m[1] - 0.3 / np.sqrt(2)) < 5e-3
    assert abs(m[2] - st) < 1e-4


def test_strouhal_needs_two_full_periods():
    t = np.linspace(0.0, 10.0, 1001)
    m = qoi.cylinder_qoi(t, np.ones_like(t), np.sin(0.2 * t), 0.2, 0.0)
    assert np.isnan(m[2])
