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


def test_cylinder_sample_qois_from_a_force_history():
    from tensum_b200 import cylinder
    mach, ang = 0.2, 2.0
    a = np.deg2rad(ang)
    q = 0.5 * mach * mach
    t = np.linspace(0.0, 40.0, 4001)
    w = 2 * np.pi * 0.5
    # drag coefficient 1.2 (0.9 inviscid + 0.3 viscous), lift 0.1 sin(w t), in the free stream's axes
    cd_i, cd_v, cl = 0.9, 0.3, 0.1 * np.sin(w * t)
    def rows(cd, cl_):
        return np.stack([(cd * np.cos(a) - cl_ * np.sin(a)) * q, (cd * np.sin(a) + cl_ * np.cos(a)) * q], axis=1)
    f = np.concatenate([rows(cd_i, cl), rows(cd_v, 0.0 * t)], axis=1)
    y = cylinder.qois(t, f, mach, ang, t_start=10.0)
    assert abs(y[0] - 1.2) < 1e-12
    assert abs(y[1] - 0.1 / np.sqrt(2)) < 1e-3
    assert abs(y[2] - 0.25) < 1e-12


def test_cylinder_inputs_are_seeded_and_in_range():
    from tensum_b200 import cylinder
    x = cylinder.draw_inputs(4096, 7)
    assert np.array_equal(x, cylinder.draw_inputs(4096, 7)) and not np.array_equal(x, cylinder.draw_inputs(4096, 8))
    lo, hi = np.array([0.15, 80.0, -2.0]), np.array([0.25, 120.0, 2.0])
    assert np.all(x >= lo) and np.all(x <= hi)
    assert np.all(np.abs(x.mean(axis=0) - (lo + hi) / 2) < 0.02 * (hi - lo))
