"""Cylinder quantities of interest from the force history.

The forces are those compute_forces reports (src/force.cc:116-219): the
pressure and viscous integrals over the cylinder's faces.  Drag and lift are
their components along and across the free stream, scaled by the dynamic head
0.5 rho U^2 D; the QoIs of the cylinder configurations are the time-averaged
drag, the root mean square of the lift fluctuation and the Strouhal number of
the shedding, f D / U from the lift's upward zero crossings.
"""
from __future__ import annotations

import numpy as np


def force_coefficients(force_rows, mach: float, angle_deg: float, rho: float = 1.0, diameter: float = 1.0):
    """(drag, lift) coefficients from rows (inviscid x, y, viscous x, y)."""
    f = np.atleast_2d(np.asarray(force_rows, np.float64))
    fx, fy = f[:, 0] + f[:, 2], f[:, 1] + f[:, 3]
    a = np.deg2rad(angle_deg)
    q = 0.5 * rho * mach * mach * diameter
    return (fx * np.cos(a) + fy * np.sin(a)) / q, (-fx * np.sin(a) + fy * np.cos(a)) / q


def cylinder_qoi(times, cd, cl, mach: float, t_start: float, diameter: float = 1.0) -> np.ndarray:
    """(mean drag, lift fluctuation RMS, Strouhal number) over t >= t_start;
    the Strouhal number is NaN when fewer than two full lift periods fall in the window."""
    t = np.asarray(times, np.float64)
    sel = t >= t_start
    t, cd, cl = t[sel], np.asarray(cd)[sel], np.asarray(cl)[sel]
    mean_cd = float(np.mean(cd))
    fl = cl - np.mean(cl)
    rms = float(np.sqrt(np.mean(fl * fl)))
    up = np.nonzero((fl[:-1] < 0.0) & (fl[1:] >= 0.0))[0]
    st = np.nan
    if up.size >= 3:
        # linear interpolation of the crossing times
        tc = t[up] - fl[up] * (t[up + 1] - t[up]) / (fl[up + 1] - fl[up])
        st = float(diameter / (np.mean(np.diff(tc)) * mach))
    return np.array([mean_cd, rms, st])
