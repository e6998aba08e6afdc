"""ctypes mirror of the C ABI structs in include/tensum_gpu.h.

Host-side glue only: builds ``tg_mesh`` / ``tg_material`` / ``tg_bc_table`` /
``tg_options`` from numpy arrays and keeps those arrays alive for as long as
the struct is in use.
"""
from __future__ import annotations

import ctypes as C
import dataclasses

import numpy as np

from .preproc import Geometry

dp = C.POINTER(C.c_double)
ip = C.POINTER(C.c_int)
bp = C.POINTER(C.c_ubyte)

FLUX = {"kepes_tecno_roe": 0, "kepes_tecno_rusanov": 1, "kepec": 2, "roe_ec": 3, "kep": 4, "simple_avg": 5}
RECON = {"first": 0, "second": 1, "second_muscl": 2, "van_albada": 3, "minmod": 4, "tvb_minmod": 5, "eno2": 6}
BC = {"none": 0, "slip": 1, "noslip": 2, "farfield": 3, "inlet": 4, "outlet": 5, "pressure": 6, "periodic": 7}
STATUS = {0: "TG_OK", 1: "TG_BAD_STATE", 2: "TG_TIMEOUT", 3: "TG_CUDA_ERROR", 4: "TG_INVALID_ARG",
          5: "TG_NOT_SUPPORTED", 6: "TG_NO_DEVICE"}


class TgMesh(C.Structure):
    _fields_ = [("n_vertex", C.c_int), ("coords", dp), ("dcarea", dp), ("mcarea", dp),
                ("n_cell", C.c_int), ("cell_vertex", ip), ("cell_normal", dp), ("cell_area", dp),
                ("n_face", C.c_int), ("face_vertex", ip), ("face_type", ip), ("face_normal", dp),
                ("face_lcell", ip), ("face_rcell", ip),
                ("n_bface", C.c_int), ("bface_vertex", ip), ("bface_type", ip), ("bface_normal", dp),
                ("bface_lcell", ip), ("bface_periodic", bp),
                ("n_periodic", C.c_int), ("periodic_offsets", ip), ("periodic_members", ip),
                ("vertex_radius", dp), ("face_radius", dp), ("cell_radius", dp)]


class TgMaterial(C.Structure):
    _fields_ = [("gamma", C.c_double), ("gas_const", C.c_double), ("prandtl", C.c_double),
                ("mu_ref", C.c_double), ("T_0", C.c_double), ("T_ref", C.c_double), ("omega", C.c_double),
                ("ev_mod_alpha", C.c_double), ("ev_mod_beta", C.c_double), ("tvb_minmod_coef", C.c_double),
                ("model", C.c_int), ("flux_scheme", C.c_int), ("mu_model", C.c_int),
                ("reconstruct_scheme", C.c_int), ("nd_active", C.c_int), ("visc_active", C.c_int),
                ("heat_active", C.c_int)]


class TgBcTable(C.Structure):
    _fields_ = [("n_types", C.c_int), ("type_tag", ip), ("kind", ip), ("adiabatic", bp), ("bface_values", dp)]


class TgOptions(C.Structure):
    _fields_ = [("time_scheme", C.c_int), ("time_mode", C.c_int), ("time_step", C.c_double),
                ("cfl", C.c_double), ("final_time", C.c_double), ("n_time_stamps", C.c_int),
                ("max_iter", C.c_long), ("min_residue", C.c_double), ("bad_state_check", C.c_int),
                ("liou_fix", C.c_int), ("bc_strong", C.c_int)]


def _p(a: np.ndarray, t):
    return a.ctypes.data_as(t)


def bface_values(g: Geometry, boundary: dict) -> np.ndarray:
    """(n_bface, 2, 5) values of tg_bc_table.bface_values: T, u, v, w, p at both
    vertices of every reference boundary face, from constant boundary specs
    {tag: (kind, {"temperature": ..., "xvelocity": ..., ...})}."""
    vals = np.zeros((g.n_bface, 2, 5))
    for tag, (_, spec) in sorted(boundary.items()):
        sel = g.bface_type == int(tag)
        for j, name in enumerate(("temperature", "xvelocity", "yvelocity", "zvelocity", "pressure")):
            if name in spec:
                vals[sel, :, j] = float(spec[name])
    return vals


@dataclasses.dataclass
class Problem:
    """Everything tg_create needs, as numpy arrays plus the ctypes structs over them."""

    geom: Geometry
    cfg: dict
    keep: list = dataclasses.field(default_factory=list)

    def __post_init__(self):
        g = self.geom
        cfg = self.cfg
        k = self.keep

        def arr(a, dt):
            a = np.ascontiguousarray(a, dtype=dt)
            k.append(a)
            return a

        offs = np.zeros(len(g.periodic_sets) + 1, np.int32)
        offs[1:] = np.cumsum([len(s) for s in g.periodic_sets]) if g.periodic_sets else []
        mem = np.array([v for s in g.periodic_sets for v in s], np.int32)
        m = TgMesh()
        m.n_vertex = g.n_vertex
        m.coords = _p(arr(g.coords, np.float64), dp)
        m.dcarea = _p(arr(g.dcarea, np.float64), dp)
        m.mcarea = _p(arr(g.mcarea, np.float64), dp)
        m.n_cell = g.n_cell
        m.cell_vertex = _p(arr(g.cells, np.int32), ip)
        m.cell_normal = _p(arr(g.cell_normal, np.float64), dp)
        m.cell_area = _p(arr(g.cell_area, np.float64), dp)
        m.n_face = g.n_face
        m.face_vertex = _p(arr(g.face_vertex, np.int32), ip)
        m.face_type = _p(arr(g.face_type, np.int32), ip)
        m.face_normal = _p(arr(g.face_normal, np.float64), dp)
        m.face_lcell = _p(arr(g.face_lcell, np.int32), ip)
        m.face_rcell = _p(arr(g.face_rcell, np.int32), ip)
        m.n_bface = g.n_bface
        m.bface_vertex = _p(arr(g.bface_vertex, np.int32), ip)
        m.bface_type = _p(arr(g.bface_type, np.int32), ip)
        m.bface_normal = _p(arr(g.bface_normal, np.float64), dp)
        m.bface_lcell = _p(arr(g.bface_lcell, np.int32), ip)
        m.bface_periodic = _p(arr(g.bface_periodic, np.uint8), bp)
        m.n_periodic = len(g.periodic_sets)
        m.periodic_offsets = _p(arr(offs, np.int32), ip)
        m.periodic_members = _p(arr(mem if mem.size else np.zeros(1, np.int32), np.int32), ip)
        if g.vertex_radius is not None:   # axisymmetric
            m.vertex_radius = _p(arr(g.vertex_radius, np.float64), dp)
            m.face_radius = _p(arr(g.face_radius, np.float64), dp)
            m.cell_radius = _p(arr(g.cell_radius, np.float64), dp)
        self.mesh = m

        mat = TgMaterial()
        mat.gamma = cfg.get("gamma", 1.4)
        mat.gas_const = cfg.get("gas_const", 1.0)
        mat.prandtl = cfg.get("prandtl", 0.72)
        mat.mu_ref = cfg.get("mu_ref", 0.0)
        mat.T_0 = cfg.get("T_0", 0.0)
        mat.T_ref = cfg.get("T_ref", 1.0)
        mat.omega = cfg.get("omega", 1.0)
        mat.ev_mod_alpha = cfg.get("ev_alpha", 0.0)
        mat.ev_mod_beta = cfg.get("ev_beta", 0.0)
        mat.tvb_minmod_coef = cfg.get("tvb_M", 0.0)
        mat.model = 1 if cfg.get("model", "euler") == "ns" else 0
        mat.flux_scheme = FLUX[cfg.get("flux", "kepes_tecno_roe")]
        mat.mu_model = 0
        mat.reconstruct_scheme = RECON[cfg.get("reconstruct", "minmod")]
        mat.nd_active = 1
        mat.visc_active = 1
        mat.heat_active = 1
        self.material = mat

        # boundary table: per tag kind / adiabatic, values per bface vertex
        tags, kinds, adiab = [], [], []
        for tag, (btype, spec) in sorted(cfg["boundary"].items()):
            tags.append(int(tag))
            kinds.append(BC[btype])
            adiab.append(1 if btype in ("slip",) or (btype == "noslip" and "temperature" not in spec) else 0)
        vals = bface_values(g, cfg["boundary"])
        bc = TgBcTable()
        bc.n_types = len(tags)
        bc.type_tag = _p(arr(np.array(tags), np.int32), ip)
        bc.kind = _p(arr(np.array(kinds), np.int32), ip)
        bc.adiabatic = _p(arr(np.array(adiab), np.uint8), bp)
        bc.bface_values = _p(arr(vals.reshape(-1) if vals.size else np.zeros(1), np.float64), dp)
        self.bc = bc

        o = TgOptions()
        o.time_scheme = {"ssprk3": 0, "rk4": 1, "heuns": 2}[cfg.get("time_scheme", "ssprk3")]
        o.time_mode = 1 if cfg.get("time_mode", "unsteady") == "unsteady" else 0
        o.time_step = cfg.get("time_step", 0.0)
        o.cfl = cfg.get("cfl", 0.8)
        o.final_time = cfg.get("final_time", 10.0)
        o.n_time_stamps = cfg.get("time_stamps", 1)
        o.max_iter = cfg.get("max_iter", 1000000000)
        o.min_residue = 0.0
        o.bad_state_check = 1
        o.liou_fix = 1 if cfg.get("liou_fix", False) else 0
        o.bc_strong = 1 if cfg.get("bc_scheme", "weak") == "strong" else 0
        self.options = o
