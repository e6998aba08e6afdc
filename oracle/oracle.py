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
        L.tor_counter.argtypes = [vp]
        L.tor_get_residual.argtypes = [vp, dp]
        L.tor_forces.argtypes = [vp, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), dp]
        L.tor_moment_nvars.argtypes = [C.c_int]
        L.tor_moments_increment.argtypes = [vp, C.c_long, C.c_int, dp, dp, dp]
        L.tor_moments_merge.argtypes = [C.c_int, C.c_int, C.c_long, dp, dp, dp, C.c_long, dp, dp, dp]
        L.tor_moments_merge.restype = C.c_long
        L.tor_moments_finalize.argtypes = [C.c_int, C.c_int, C.c_long, dp, dp]
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

    def current_residual(self):
        out = np.empty((self.nv, 5))
        self.L.tor_get_residual(self.h, _d(out))
        return out

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

    def forces(self, forces: dict) -> np.ndarray:
        """compute_forces for {name: [tags]} (insertion order): rows inviscid x, y, viscous x, y."""
        n = np.array([len(t) for t in forces.values()], np.int32)
        tags = np.array([x for t in forces.values() for x in t], np.int32)
        out = np.empty((len(n), 4))
        ip = C.POINTER(C.c_int)
        self.L.tor_forces(self.h, len(n), n.ctypes.data_as(ip), tags.ctypes.data_as(ip), _d(out))
        return out

    def global_integrals(self):
        a = C.c_double()
        b = C.c_double()
        self.L.tor_global(self.h, C.byref(a), C.byref(b))
        return a.value, b.value


def moment_nvars(extras: int) -> int:
    return lib().tor_moment_nvars(extras)


def moments_merge(n_old, fm, sm, m2, n_other, fm_o, sm_o, m2_o):
    """reduce_moments' merge of one received group into (fm, sm, m2), in place; returns the new count."""
    nv, nvar = fm.shape
    return lib().tor_moments_merge(nv, nvar, n_old, _d(fm), _d(sm), _d(m2), n_other,
                                   _d(np.ascontiguousarray(fm_o)), _d(np.ascontiguousarray(sm_o)),
                                   _d(np.ascontiguousarray(m2_o)))


def moments_finalize(n, sm, m2):
    nv, nvar = sm.shape
    lib().tor_moments_finalize(nv, nvar, n, _d(sm), _d(m2))


def run_mc(problem, ics, n_instances: int, extras: int):
    """The reference's per-group Monte Carlo loop (src/fv.cc:2401-2466 with
    solve's increment_moments calls, src/fv.cc:2230-2380) over the given
    initial states, unsteady mode.  Returns the raw (unscaled) group moments
    fm, sm, m2 of shape (n_instances, n_vertex, nvars)."""
    o = Oracle(problem)
    L = o.L
    nvar = L.tor_moment_nvars(extras)
    shape = (n_instances, o.nv, nvar)
    fm, sm, m2 = np.zeros(shape), np.zeros(shape), np.zeros(shape)
    for k, ic in enumerate(ics, 1):
        o.set_prim(ic)
        L.tor_compute_gradients(o.h, None)       # solve() starts with compute_gradients
        L.tor_moments_increment(o.h, k, extras, _d(fm[0]), _d(sm[0]), _d(m2[0]))
        for t in range(1, n_instances):
            while L.tor_counter(o.h) <= t:
                done, _ = o.step(1)
                if done == 0:
                    raise RuntimeError("oracle run ended before output instance %d" % t)
            L.tor_moments_increment(o.h, k, extras, _d(fm[t]), _d(sm[t]), _d(m2[t]))
    return fm, sm, m2
