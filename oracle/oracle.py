"""ctypes wrapper of the C restatement (oracle/_build/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py as the checker.  The product path never imports
this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")
_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
    return LIB


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        vp = C.c_void_p
        dp = C.POINTER(C.c_double)
        L.tor_create.restype = vp
        L.tor_create.argtypes = [vp, vp, vp, vp]
        L.tor_destroy.argtypes = [vp]
        L.tor_n_vertex.argtypes = [vp]
        L.tor_set_prim.argtypes = [vp, dp, C.c_double]
        L.tor_get_prim.argtypes = [vp, dp]
        L.tor_store_conserved_old.argtypes = [vp]
        L.tor_compute_dt.argtypes = [vp, dp]
        L.tor_compute_dt.restype = C.c_double
        L.tor_compute_gradients.argtypes = [vp, dp]
        L.tor_compute_residual.argtypes = [vp, dp, dp]
        L.tor_update.argtypes = [vp, C.c_int]
        L.tor_residual_norm.argtypes = [vp, C.c_long, dp]
        L.tor_end_step.argtypes = [vp]
        L.tor_step.argtypes = [vp, C.c_long, dp]
        L.tor_step.restype = C.c_long
        L.tor_global.argtypes = [vp, dp, dp]
        L.tor_num_flux.argtypes = [vp] + [dp] * 8
        L.tor_logavg.argtypes = [C.c_double, C.c_double]
        L.tor_logavg.restype = C.c_double
        _lib = L
    return _lib


def _d(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Oracle:
    """One reference-equivalent CPU solver instance over a tensum_b200.abi.Problem."""

    def __init__(self, problem):
        self.problem = problem  # keeps arrays alive
        L = lib()
        self.L = L
        self.h = L.tor_create(C.byref(problem.mesh), C.byref(problem.material), C.byref(problem.bc),
                              C.byref(problem.options))
        self.nv = problem.geom.n_vertex

    def __del__(self):
        try:
            if self.h:
                self.L.tor_destroy(self.h)
        except Exception:
            pass

    def set_prim(self, prim, t0=0.0):
        prim = np.ascontiguousarray(prim, np.float64)
        self.L.tor_set_prim(self.h, _d(prim), t0)

    def get_prim(self):
        out = np.empty((self.nv, 5))
        self.L.tor_get_prim(self.h, _d(out))
        return out

    def store_conserved_old(self):
        self.L.tor_store_conserved_old(self.h)

    def compute_dt(self):
        dt = np.empty(self.nv)
        g = self.L.tor_compute_dt(self.h, _d(dt))
        return g, dt

    def gradients(self):
        out = np.empty((self.nv, 5, 3))
        self.L.tor_compute_gradients(self.h, _d(out))
        return out

    def residual(self):
        res = np.empty((self.nv, 5))
        dE = np.empty((self.nv, 5, 3))
        self.L.tor_compute_residual(self.h, _d(res), _d(dE))
        return res, dE

    def update(self, r):
        self.L.tor_update(self.h, r)

    def residual_norm(self, it):
        out = np.empty(6)
        self.L.tor_residual_norm(self.h, it, _d(out))
        return out

    def end_step(self):
        self.L.tor_end_step(self.h)

    def step(self, n):
        info = np.empty(4)
        done = self.L.tor_step(self.h, n, _d(info))
        return done, info

    def global_integrals(self):
        a = C.c_double()
        b = C.c_double()
        self.L.tor_global(self.h, C.byref(a), C.byref(b))
        return a.value, b.value
