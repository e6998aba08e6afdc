"""ctypes binding of the batched FP32 ensembles (tg_batch_* in include/tensum_gpu.h).

    from tensum_b200 import abi, batch, cases, preproc
    P = abi.Problem(preproc.preprocess(cases.kh_mesh(257, 0)), cfg)
    b = batch.Batch([(P, 4096)])
    b.set_kh(0, rows)                  # rows: (4096, 20) random numbers per sample
    b.tune(3)                          # autotuner: pick the fastest launch shape
    b.advance(1)                       # every sample to output time 1
    fm, sm, m2 = b.moments(0, extras=1)
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi, gpu


class tg_batch_level(C.Structure):
    _fields_ = [("mesh", C.c_void_p), ("bc", C.c_void_p), ("n_samples", C.c_int)]


_bound = False


def _lib():
    global _bound
    L = gpu.load()
    if not _bound:
        vp, i, dp, ip = C.c_void_p, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_int)
        L.tg_batch_create.argtypes = [C.POINTER(tg_batch_level), i, vp, vp, C.POINTER(vp)]
        L.tg_batch_destroy.argtypes = [vp]
        L.tg_batch_last_error.argtypes = [vp]
        L.tg_batch_last_error.restype = C.c_char_p
        L.tg_batch_set_state.argtypes = [vp, i, i, dp, i]
        L.tg_batch_get_state.argtypes = [vp, i, i, dp, i]
        L.tg_batch_set_kh.argtypes = [vp, i, dp, i]
        L.tg_batch_advance.argtypes = [vp, i, C.c_long, dp]
        L.tg_batch_clock.argtypes = [vp, i, dp, ip, ip]
        L.tg_batch_moments.argtypes = [vp, i, i, dp, dp, dp]
        L.tg_batch_set_shape.argtypes = [vp, i]
        L.tg_batch_tune.argtypes = [vp, i, ip, dp]
        L.tg_batch_time_steps.argtypes = [vp, i, dp]
        L.tg_batch_stream.argtypes = [vp, C.POINTER(vp)]
        L.tg_batch_query.argtypes = [vp, i, dp]
        L.tg_batch_integrals.argtypes = [vp, i, dp]
        L.tg_batch_set_parameters.argtypes = [vp, i, dp, dp]
        L.tg_batch_set_uniform.argtypes = [vp, i, dp]
        L.tg_batch_forces.argtypes = [vp, i, i, ip, ip, dp]
        L.tg_batch_set_state_expr.argtypes = [vp, i, C.POINTER(vp), dp, i]
        L.tg_batch_set_bc_expr.argtypes = [vp, i, i, C.POINTER(vp), dp, i, C.c_double]
        for n in ("tg_batch_create", "tg_batch_destroy", "tg_batch_set_state", "tg_batch_get_state",
                  "tg_batch_set_kh", "tg_batch_advance", "tg_batch_clock", "tg_batch_moments",
                  "tg_batch_set_shape", "tg_batch_tune", "tg_batch_time_steps", "tg_batch_stream",
                  "tg_batch_query", "tg_batch_integrals", "tg_batch_set_parameters", "tg_batch_set_uniform",
                  "tg_batch_forces", "tg_batch_set_state_expr", "tg_batch_set_bc_expr"):
            getattr(L, n).restype = i
        _bound = True
    return L


def _d(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


QUERY = {"n_levels": 0, "kernels_per_step": 1, "device_bytes": 2, "shape": 3, "sample_tile": 4, "block": 5,
         "n_shapes": 6}


class Batch:
    """An ensemble batch of one or more (problem, n_samples) levels."""

    def __init__(self, levels):
        self.L = _lib()
        self.problems = [p for p, _ in levels]
        self.S = [int(n) for _, n in levels]
        arr = (tg_batch_level * len(levels))()
        for j, (p, n) in enumerate(levels):
            arr[j].mesh = C.cast(C.pointer(p.mesh), C.c_void_p)
            arr[j].bc = C.cast(C.pointer(p.bc), C.c_void_p)
            arr[j].n_samples = int(n)
        p0 = self.problems[0]
        h = C.c_void_p()
        st = self.L.tg_batch_create(arr, len(levels), C.byref(p0.material), C.byref(p0.options), C.byref(h))
        if st != 0:
            raise gpu.TensumError(st, self.L.tg_batch_last_error(None).decode())
        self.h = h
        self.nv = [p.geom.n_vertex for p in self.problems]

    def __del__(self):
        try:
            if getattr(self, "h", None):
                self.L.tg_batch_destroy(self.h)
                self.h = None
        except Exception:
            pass

    def _chk(self, st):
        if st != 0:
            raise gpu.TensumError(st, self.L.tg_batch_last_error(self.h).decode())

    def set_state(self, level: int, sample: int, prim: np.ndarray):
        prim = np.ascontiguousarray(prim, np.float64)
        self._chk(self.L.tg_batch_set_state(self.h, level, sample, _d(prim), self.nv[level]))

    def get_state(self, level: int, sample: int) -> np.ndarray:
        out = np.empty((self.nv[level], 5))
        self._chk(self.L.tg_batch_get_state(self.h, level, sample, _d(out), self.nv[level]))
        return out

    def set_kh(self, level: int, rows: np.ndarray):
        rows = np.ascontiguousarray(rows, np.float64)
        assert rows.shape[0] == self.S[level]
        self._chk(self.L.tg_batch_set_kh(self.h, level, _d(rows), rows.shape[1]))

    def set_parameters(self, level: int, mu_ref=None, bface_values=None):
        """Per-sample viscosity (S,) and boundary values (S, n_bface, 2, 5) of a level
        with boundary faces or viscosity; None keeps the current ones."""
        S = self.S[level]
        mu = None if mu_ref is None else np.ascontiguousarray(mu_ref, np.float64).reshape(S)
        bv = None
        if bface_values is not None:
            bv = np.ascontiguousarray(bface_values, np.float64)
            assert bv.shape[0] == S and bv.size == S * self.problems[level].geom.n_bface * 10
        self._chk(self.L.tg_batch_set_parameters(self.h, level, None if mu is None else _d(mu),
                                                 None if bv is None else _d(bv)))

    def set_uniform(self, level: int, prim: np.ndarray):
        """Every sample at its own uniform PrimVar record prim[s] = (T, p, u, v, w)."""
        prim = np.ascontiguousarray(prim, np.float64)
        assert prim.shape == (self.S[level], 5)
        self._chk(self.L.tg_batch_set_uniform(self.h, level, _d(prim)))

    def set_state_expr(self, level: int, fields, rnd_rows=None):
        """Every sample's initial state from expressions (gpu.expr_fields), sample s
        with random numbers rnd_rows[s], evaluated on the device."""
        S = self.S[level]
        r = np.ascontiguousarray(rnd_rows if rnd_rows is not None else np.zeros((S, 0)), np.float64)
        assert r.shape[0] == S
        self._chk(self.L.tg_batch_set_state_expr(self.h, level, gpu.expr_array(fields), _d(r) if r.size else None,
                                                 r.shape[1]))

    def set_bc_expr(self, level: int, tag: int, fields, rnd_rows=None, t: float = 0.0):
        """Per-sample boundary values of the faces of `tag` from expressions (None keeps a variable)."""
        S = self.S[level]
        r = np.ascontiguousarray(rnd_rows if rnd_rows is not None else np.zeros((S, 0)), np.float64)
        assert r.shape[0] == S
        self._chk(self.L.tg_batch_set_bc_expr(self.h, level, tag, gpu.expr_array(fields), _d(r) if r.size else None,
                                              r.shape[1], t))

    def forces(self, level: int, forces: dict) -> np.ndarray:
        """(S, n_forces, 4): compute_forces of every sample for {name: [face tags]}."""
        n = np.array([len(t) for t in forces.values()], np.int32)
        tags = np.array([x for t in forces.values() for x in t], np.int32)
        out = np.empty((self.S[level], len(n), 4))
        ip = C.POINTER(C.c_int)
        self._chk(self.L.tg_batch_forces(self.h, level, len(n), n.ctypes.data_as(ip), tags.ctypes.data_as(ip), _d(out)))
        return out

    def advance(self, instance: int, max_steps: int = 1 << 40) -> np.ndarray:
        info = np.empty(4)
        self._chk(self.L.tg_batch_advance(self.h, instance, max_steps, _d(info)))
        return info

    def clock(self, level: int):
        S = self.S[level]
        el, cnt, bad = np.empty(S), np.empty(S, np.int32), np.empty(S, np.int32)
        self._chk(self.L.tg_batch_clock(self.h, level, _d(el), cnt.ctypes.data_as(C.POINTER(C.c_int)),
                                        bad.ctypes.data_as(C.POINTER(C.c_int))))
        return el, cnt, bad

    def moments(self, level: int, extras: int = 0):
        nvar = 5 + bin(extras).count("1")
        out = [np.empty((self.nv[level], nvar)) for _ in range(3)]
        self._chk(self.L.tg_batch_moments(self.h, level, extras, *[_d(a) for a in out]))
        return out

    def integrals(self, level: int) -> np.ndarray:
        """(n_samples, 3): 0.5 rho v^2, 0.5 rho u^2 and -rho s/(gamma-1) integrated over the mesh."""
        out = np.empty((self.S[level], 3))
        self._chk(self.L.tg_batch_integrals(self.h, level, _d(out)))
        return out

    def set_shape(self, shape: int):
        self._chk(self.L.tg_batch_set_shape(self.h, shape))

    def tune(self, steps: int = 3):
        n = int(self.query("n_shapes"))
        ms = np.empty(n)
        best = C.c_int()
        self._chk(self.L.tg_batch_tune(self.h, steps, C.byref(best), _d(ms)))
        return best.value, ms

    def time_steps(self, steps: int) -> float:
        ms = C.c_double()
        self._chk(self.L.tg_batch_time_steps(self.h, steps, C.byref(ms)))
        return ms.value

    def stream_ptr(self) -> int:
        p = C.c_void_p()
        self._chk(self.L.tg_batch_stream(self.h, C.byref(p)))
        return p.value or 0

    def query(self, key: str) -> float:
        out = C.c_double()
        self._chk(self.L.tg_batch_query(self.h, QUERY[key], C.byref(out)))
        return out.value
