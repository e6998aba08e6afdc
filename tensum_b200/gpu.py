"""Python binding of the C ABI (include/tensum_gpu.h) via ctypes.

The device library is mandatory: loading fails loudly if it is missing, and
:class:`Solver` raises if ``tg_create`` reports no CUDA device.  There is no
CPU fallback anywhere on this path.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import abi

HERE = os.path.dirname(os.path.abspath(__file__))
# TENSUM_B200_LIB selects another build of the library (e.g. one with other tile sizes)
LIB_PATH = os.environ.get("TENSUM_B200_LIB") or os.path.join(HERE, "libtensum_b200.so")

EXPORTS = ["tg_create", "tg_destroy", "tg_last_error", "tg_abi_version", "tg_set_state", "tg_get_state",
           "tg_store_conserved_old", "tg_compute_dt", "tg_gradients", "tg_residual", "tg_update",
           "tg_residual_norm", "tg_end_step", "tg_step", "tg_global", "tg_stream", "tg_time_phase", "tg_query",
           "tg_advance", "tg_moments_init", "tg_moments_increment", "tg_moments_get", "tg_moments_export",
           "tg_moments_merge", "tg_moments_merge_device", "tg_moments_finalize", "tg_forces", "tg_update_parameters",
           "tg_output_begin", "tg_output_wait", "tg_set_state_async", "tg_expr_create", "tg_expr_destroy",
           "tg_expr_last_error", "tg_expr_eval", "tg_set_state_expr", "tg_part_plan", "tg_part_create",
           "tg_part_info", "tg_part_prime", "tg_part_begin", "tg_part_gradients", "tg_part_flux", "tg_part_pack",
           "tg_part_unpack", "tg_part_export", "tg_part_import", "tg_part_scalars"]

ABI_VERSION = 4        # TG_ABI_VERSION of include/tensum_gpu.h
PHASE = {"gradient": 0, "flux": 1, "update": 2, "dt": 3, "step": 4}
QUERY = {"n_vertex": 0, "n_edge": 1, "n_bface": 2, "kernels_per_step": 3, "device_bytes": 4, "kernels_per_flux": 5,
         "n_tiles": 6}

_lib = None


class TensumError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{abi.STATUS.get(status, status)}: {msg}")
        self.status = status


def load():
    """Load libtensum_b200.so (raises OSError when it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise OSError(f"{LIB_PATH} is missing; build it with `python -m tensum_b200.build`")
    L = C.CDLL(LIB_PATH)
    vp, dp, i = C.c_void_p, C.POINTER(C.c_double), C.c_int
    L.tg_create.argtypes = [vp, vp, vp, vp, C.POINTER(vp)]
    L.tg_destroy.argtypes = [vp]
    L.tg_last_error.argtypes = [vp]
    L.tg_last_error.restype = C.c_char_p
    L.tg_abi_version.restype = i
    L.tg_set_state.argtypes = [vp, dp, i, C.c_double]
    L.tg_get_state.argtypes = [vp, dp, i]
    L.tg_store_conserved_old.argtypes = [vp]
    L.tg_compute_dt.argtypes = [vp, dp, dp]
    L.tg_gradients.argtypes = [vp, dp]
    L.tg_residual.argtypes = [vp, dp]
    L.tg_update.argtypes = [vp, i]
    L.tg_residual_norm.argtypes = [vp, C.c_long, dp]
    L.tg_end_step.argtypes = [vp, dp]
    L.tg_step.argtypes = [vp, i, dp]
    L.tg_global.argtypes = [vp, dp, dp]
    L.tg_stream.argtypes = [vp, C.POINTER(vp)]
    L.tg_time_phase.argtypes = [vp, i, i, dp]
    L.tg_query.argtypes = [vp, i, dp]
    L.tg_advance.argtypes = [vp, i, C.c_long, dp]
    L.tg_forces.argtypes = [vp, i, C.POINTER(i), C.POINTER(i), dp]
    L.tg_update_parameters.argtypes = [vp, vp, vp]
    L.tg_output_begin.argtypes = [vp, dp, dp, i]
    L.tg_output_wait.argtypes = [vp]
    L.tg_set_state_async.argtypes = [vp, dp, i, C.c_double]
    L.tg_expr_create.argtypes = [C.c_char_p, i, C.POINTER(C.c_char_p), dp, C.POINTER(vp)]
    L.tg_expr_destroy.argtypes = [vp]
    L.tg_expr_last_error.argtypes = []
    L.tg_expr_last_error.restype = C.c_char_p
    L.tg_expr_eval.argtypes = [vp, C.c_double, C.c_double, C.c_double, dp, i, dp]
    L.tg_set_state_expr.argtypes = [vp, C.POINTER(vp), dp, i, C.c_double]
    L.tg_moments_init.argtypes = [vp, i, i]
    L.tg_moments_increment.argtypes = [vp, i, C.c_long]
    L.tg_moments_get.argtypes = [vp, i, dp, dp, dp]
    L.tg_moments_export.argtypes = [vp, i, vp]
    L.tg_moments_merge.argtypes = [vp, i, C.c_long, C.c_long, dp, dp, dp]
    L.tg_moments_merge_device.argtypes = [vp, i, C.c_long, C.c_long, vp]
    L.tg_moments_finalize.argtypes = [vp, i, C.c_long]
    ip = C.POINTER(i)
    L.tg_part_plan.argtypes = [vp, vp, i, i, ip, ip, ip, ip, ip, ip]
    L.tg_part_create.argtypes = [vp, vp, vp, vp, i, i, C.POINTER(vp)]
    L.tg_part_info.argtypes = [vp, ip, ip, ip]
    for name in ("tg_part_prime", "tg_part_begin"):
        getattr(L, name).argtypes = [vp]
    L.tg_part_gradients.argtypes = [vp, i, i]
    L.tg_part_flux.argtypes = [vp, i, i]
    L.tg_part_pack.argtypes = [vp, i, vp]
    L.tg_part_unpack.argtypes = [vp, i, vp]
    L.tg_part_export.argtypes = [vp, vp]
    L.tg_part_import.argtypes = [vp, vp]
    L.tg_part_scalars.argtypes = [vp, dp]
    for name in EXPORTS:
        f = getattr(L, name)
        if name not in ("tg_last_error", "tg_abi_version", "tg_expr_last_error"):
            f.restype = i
    if L.tg_abi_version() != ABI_VERSION:
        raise OSError(f"{LIB_PATH} has ABI version {L.tg_abi_version()}, this binding needs {ABI_VERSION}; "
                      "rebuild it with `python -m tensum_b200.build`")
    _lib = L
    return L


def _d(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Expr:
    """A parameter-file expression of (x, y, t) compiled for host and device
    evaluation (tg_expr_*): fparser syntax, pi, the given named constants and
    pert(type, x, y, p) over a sample's random numbers."""

    def __init__(self, text: str, constants: dict | None = None):
        self.L = load()
        consts = dict(constants or {})
        names = (C.c_char_p * max(1, len(consts)))(*[k.encode() for k in consts])
        vals = np.array(list(consts.values()) or [0.0], np.float64)
        h = C.c_void_p()
        st = self.L.tg_expr_create(text.encode(), len(consts), names, _d(vals), C.byref(h))
        if st != 0:
            raise TensumError(st, self.L.tg_expr_last_error().decode())
        self.h = h
        self.text = text

    def __del__(self):
        try:
            if getattr(self, "h", None):
                self.L.tg_expr_destroy(self.h)
                self.h = None
        except Exception:
            pass

    def __call__(self, x: float, y: float, t: float = 0.0, rnd=None) -> float:
        r = np.ascontiguousarray(rnd if rnd is not None else np.zeros(1), np.float64)
        out = C.c_double()
        st = self.L.tg_expr_eval(self.h, float(x), float(y), float(t), _d(r), 0 if rnd is None else r.size,
                                 C.byref(out))
        if st != 0:
            raise TensumError(st, self.L.tg_expr_last_error().decode())
        return out.value


def expr_fields(ic: dict, constants: dict | None = None):
    """Five Expr (temperature, x/y/z velocity, pressure; z velocity may be absent)
    from {variable: expression} as the initial_condition section names them."""
    names = ("temperature", "xvelocity", "yvelocity", "zvelocity", "pressure")
    return [Expr(ic[n], constants) if n in ic else None for n in names]


def expr_array(fields):
    vp = C.c_void_p
    return (vp * 5)(*[f.h if f is not None else None for f in fields])


class Solver:
    """One device solver instance (mirrors the FiniteVolume hot-path members)."""

    def __init__(self, problem: abi.Problem):
        self.L = load()
        self.problem = problem
        self.nv = problem.geom.n_vertex
        h = C.c_void_p()
        st = self.L.tg_create(C.byref(problem.mesh), C.byref(problem.material), C.byref(problem.bc),
                              C.byref(problem.options), C.byref(h))
        if st != 0:
            raise TensumError(st, self.L.tg_last_error(None).decode())
        self.h = h

    def _chk(self, st):
        if st != 0:
            raise TensumError(st, self.L.tg_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            self.L.tg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_state(self, prim: np.ndarray, t0: float = 0.0):
        prim = np.ascontiguousarray(prim, np.float64)
        self._chk(self.L.tg_set_state(self.h, _d(prim), self.nv, t0))

    def set_state_async(self, prim: np.ndarray, t0: float = 0.0):
        """Queue a state from pinned host memory (see output_buffers); the next
        step() / advance() takes it in.  Keep the buffer unchanged until then."""
        if prim.dtype != np.float64 or not prim.flags.c_contiguous or prim.shape != (self.nv, 5):
            raise ValueError("prim must be a C-contiguous float64 array of shape (n_vertex, 5)")
        self._in_keep = getattr(self, "_in_keep", [])[-1:] + [prim]
        self._chk(self.L.tg_set_state_async(self.h, _d(prim), self.nv, t0))

    def set_state_expr(self, fields, rnd=None, t0: float = 0.0):
        """The initial condition evaluated on the device from expr_fields(...)
        with one sample's random numbers, taken in as set_state takes a state."""
        r = np.ascontiguousarray(rnd if rnd is not None else np.zeros(1), np.float64)
        self._chk(self.L.tg_set_state_expr(self.h, expr_array(fields), _d(r), 0 if rnd is None else r.size, t0))

    def get_state(self, out: np.ndarray | None = None) -> np.ndarray:
        """The state as (n_vertex, 5) PrimVar records; written into `out` when given
        (C-contiguous float64, e.g. a view of pinned host memory, which is copied by DMA
        without staging)."""
        if out is None:
            out = np.empty((self.nv, 5))
        elif out.shape != (self.nv, 5) or out.dtype != np.float64 or not out.flags.c_contiguous:
            raise ValueError("out must be a C-contiguous float64 array of shape (n_vertex, 5)")
        self._chk(self.L.tg_get_state(self.h, _d(out), self.nv))
        return out

    def store_conserved_old(self):
        self._chk(self.L.tg_store_conserved_old(self.h))

    def compute_dt(self):
        g = C.c_double()
        dt = np.empty(self.nv)
        self._chk(self.L.tg_compute_dt(self.h, C.byref(g), _d(dt)))
        return g.value, dt

    def gradients(self) -> np.ndarray:
        out = np.empty((self.nv, 5, 3))
        self._chk(self.L.tg_gradients(self.h, _d(out)))
        return out

    def residual(self) -> np.ndarray:
        out = np.empty((self.nv, 5))
        self._chk(self.L.tg_residual(self.h, _d(out)))
        return out

    def update(self, r: int):
        self._chk(self.L.tg_update(self.h, r))

    def residual_norm(self, it: int) -> np.ndarray:
        out = np.empty(6)
        self._chk(self.L.tg_residual_norm(self.h, it, _d(out)))
        return out

    def end_step(self) -> np.ndarray:
        info = np.empty(4)
        self._chk(self.L.tg_end_step(self.h, _d(info)))
        return info

    def step(self, n: int) -> np.ndarray:
        info = np.empty(4)
        self._chk(self.L.tg_step(self.h, n, _d(info)))
        return info

    def global_integrals(self):
        a, b = C.c_double(), C.c_double()
        self._chk(self.L.tg_global(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def update_parameters(self, problem):
        """Material constants and boundary values of `problem` (same mesh and schemes)."""
        self._keep = problem          # the ctypes structs point into its arrays
        self._chk(self.L.tg_update_parameters(self.h, C.byref(problem.material), C.byref(problem.bc)))

    # ---- output snapshots (tg_output_begin / tg_output_wait)
    GRAD_LAST_STAGE, GRAD_CURRENT = 0, 1

    def output_buffers(self, with_gradients: bool = True):
        """Pinned host buffers for output_begin: state (n_vertex, 5) and dE (n_vertex, 5, 3)."""
        import torch
        prim = torch.empty((self.nv, 5), dtype=torch.float64, pin_memory=True).numpy()
        grad = torch.empty((self.nv, 5, 3), dtype=torch.float64, pin_memory=True).numpy() if with_gradients else None
        return prim, grad

    def output_begin(self, prim_out: np.ndarray, grad_out: np.ndarray | None = None,
                     grad_state: int = GRAD_LAST_STAGE):
        """Start copying the current state (and gradients) into pinned buffers;
        later calls overlap the copy until output_wait."""
        self._out_keep = (prim_out, grad_out)
        self._chk(self.L.tg_output_begin(self.h, _d(prim_out), None if grad_out is None else _d(grad_out), grad_state))

    def output_wait(self):
        self._chk(self.L.tg_output_wait(self.h))

    def forces(self, forces: dict) -> np.ndarray:
        """compute_forces on the current state for {name: [face tags]} (in insertion
        order, like the reference's integrals section): one row per force with the
        inviscid x, y and viscous x, y components."""
        n = np.array([len(t) for t in forces.values()], np.int32)
        tags = np.array([x for t in forces.values() for x in t], np.int32)
        out = np.empty((len(n), 4))
        ip = C.POINTER(C.c_int)
        self._chk(self.L.tg_forces(self.h, len(n), n.ctypes.data_as(ip), tags.ctypes.data_as(ip), _d(out)))
        return out

    # ---- output-time stepping and Monte Carlo moments
    def advance(self, instance: int, max_steps: int = 1 << 40) -> np.ndarray:
        """Step until output time `instance` is reached; returns elapsed, dt,
        residual, iterations and the output-time counter."""
        info = np.empty(5)
        self._chk(self.L.tg_advance(self.h, instance, max_steps, _d(info)))
        return info

    def moments_init(self, n_instances: int, extras: int = 0):
        self._chk(self.L.tg_moments_init(self.h, n_instances, extras))
        self.mom_nvar = 5 + bin(extras).count("1")

    def moments_increment(self, instance: int, k: int):
        self._chk(self.L.tg_moments_increment(self.h, instance, k))

    def moments_get(self, instance: int):
        """Raw group moments (fm, sm, m2) of one instance, each (n_vertex, nvar)."""
        out = [np.empty((self.nv, self.mom_nvar)) for _ in range(3)]
        self._chk(self.L.tg_moments_get(self.h, instance, *[_d(a) for a in out]))
        return out

    def moments_export(self, instance: int, dev_ptr: int):
        self._chk(self.L.tg_moments_export(self.h, instance, C.c_void_p(dev_ptr)))

    def moments_merge(self, instance: int, n_self: int, n_other: int, fm, sm, m2):
        arrs = [np.ascontiguousarray(a, np.float64) for a in (fm, sm, m2)]
        self._chk(self.L.tg_moments_merge(self.h, instance, n_self, n_other, *[_d(a) for a in arrs]))

    def moments_merge_device(self, instance: int, n_self: int, n_other: int, dev_ptr: int):
        self._chk(self.L.tg_moments_merge_device(self.h, instance, n_self, n_other, C.c_void_p(dev_ptr)))

    def moments_finalize(self, instance: int, n: int):
        self._chk(self.L.tg_moments_finalize(self.h, instance, n))

    def stream_ptr(self) -> int:
        """cudaStream_t of this handle (for torch.cuda.ExternalStream / CUDA events)."""
        p = C.c_void_p()
        self._chk(self.L.tg_stream(self.h, C.byref(p)))
        return int(p.value or 0)

    def time_phase(self, phase: str, reps: int) -> float:
        ms = C.c_double()
        self._chk(self.L.tg_time_phase(self.h, PHASE[phase], reps, C.byref(ms)))
        return ms.value

    def query(self, key: str) -> float:
        out = C.c_double()
        self._chk(self.L.tg_query(self.h, QUERY[key], C.byref(out)))
        return out.value
