"""The reference's output files from device snapshots, byte for byte.

A drop-in run of the GPU path writes what `tensum` writes into its sample
directory.  This module restates those formats for states and gradients
brought back by `Solver.output_begin` / `output_wait` (or `get_state`):

    sol<counter>_<part>.vtk     Writer::output_vtk        src/writer.cc:129-325
    v<counter>_<part>_<tag>.dat Writer::output_surfaces   src/writer.cc:332-370
    f<counter>_<part>_<tag>.dat skin friction             src/output_skin_friction.cc:14-104
    q<counter>_<part>_<tag>.dat heat flux                 src/output_heatflux.cc:14-95
    restart_<head>_<part>.dat   Writer::output_restart    src/writer.cc:376-409
    residual.dat                log_messages              src/fv.cc:1938-1974
    force.dat                   compute_forces            src/force.cc:116-219
    global.dat                  compute_global            src/fv.cc:2175-2225

Numbers are formatted as C++ iostreams format them (default: %g with the
stream's precision; `scientific`: %e), and every derived quantity is
evaluated with the reference's operand order and libm (math.log, math.pow,
math.sqrt), so the same state gives the same text.
"""
from __future__ import annotations

import math
import os

import numpy as np

from . import abi


def _g(x: float, prec: int = 6) -> str:
    return "%.*g" % (prec, x)


def _index(counter: int) -> str:
    if counter > 9999:
        raise ValueError("counter is too large (the reference stops at 9999)")
    return "%04d" % counter


class Writer:
    """Output files of one mesh partition (part 0) for a case configuration
    (the dict abi.Problem takes: boundary, gamma, gas_const, prandtl, mu_ref, model)."""

    def __init__(self, geom, cfg: dict, part: int = 0):
        self.g = geom
        self.cfg = cfg
        self.part = part
        self.gamma = float(cfg.get("gamma", 1.4))
        self.R = float(cfg.get("gas_const", 1.0))
        self.prandtl = float(cfg.get("prandtl", 0.72))
        self.mu_ref = float(cfg.get("mu_ref", 0.0))
        self.ns = cfg.get("model", "euler") == "ns"
        self.Cp = self.gamma * self.R / (self.gamma - 1.0)   # src/material.cc:18
        # per reference boundary face: kind, adiabatic flag, values at its two vertices
        kinds, adiab = {}, {}
        for tag, (btype, spec) in cfg["boundary"].items():
            kinds[int(tag)] = abi.BC[btype]
            adiab[int(tag)] = btype == "slip" or (btype == "noslip" and "temperature" not in spec)
        self.b_kind = np.array([kinds.get(int(t), 0) for t in geom.bface_type], np.int64)
        self.b_adiab = np.array([adiab.get(int(t), False) for t in geom.bface_type], bool)
        self.b_val = abi.bface_values(geom, cfg["boundary"])

    # ------------------------------------------------------------- material
    def _density(self, T, p):
        return p / (self.R * T)                                   # src/material.h:596

    def _entropy(self, T, p):
        return math.log(p) - self.gamma * math.log(self._density(T, p))   # src/material.h:613-616

    def _mach(self, T, u, v):
        sonic = math.sqrt(self.gamma * self.R * T)                # src/material.h:585-589
        return math.sqrt(u * u + v * v + 0.0 * 0.0) / sonic

    def _viscosity(self, T):
        return self.mu_ref                                        # constant law, src/material.h:552-568

    def _prim2ent(self, T, p, u, v):                              # src/material.h:534-546
        density = self._density(T, p)
        beta = density / (2 * p)
        s = self._entropy(T, p)
        f = (self.gamma - s) / (self.gamma - 1) - (u * u + v * v + 0.0 * 0.0) * beta
        return f, u * (2 * beta), v * (2 * beta), -2 * beta

    def _bc_apply(self, b, slot, T, p, u, v):
        """Single-state BoundaryCondition::apply (src/bc.h:615-654) for face b's vertex slot."""
        kind, val = int(self.b_kind[b]), self.b_val[b, slot]
        if kind == abi.BC["slip"]:
            nx, ny = self.g.bface_normal[b]
            meas = math.sqrt(nx * nx + ny * ny + 0.0 * 0.0)
            ux, uy = nx * (1.0 / meas), ny * (1.0 / meas)
            fact = u * ux + v * uy + 0.0 * 0.0
            u, v = u + ux * -fact, v + uy * -fact
        elif kind == abi.BC["noslip"]:
            u, v = val[1], val[2]
            if not self.b_adiab[b]:
                T = val[0]
        elif kind == abi.BC["pressure"]:
            p = val[4]
        elif kind == abi.BC["inlet"]:
            T, u, v, p = val[0], val[1], val[2], val[4]
        return T, p, u, v

    # ------------------------------------------------------------------ vtk
    def vtk_text(self, prim, time=None, variables=(), dE=None) -> str:
        """Writer::output_vtk with the primitive state, the dual areas attached as
        vertex data (FiniteVolume::output) and the requested derived variables."""
        for name in variables:
            if name not in ("mach", "density", "entropy", "vorticity"):
                raise ValueError(f"unknown output variable {name!r}")
        prim = np.asarray(prim, np.float64).reshape(-1, 5)
        g = self.g
        n = g.n_vertex
        out = ["# vtk DataFile Version 3.0", "tensum", "ASCII", "DATASET UNSTRUCTURED_GRID"]
        if time is not None:
            out += ["FIELD FieldData 1", "TIME 1 1 double", _g(time)]
        out.append(f"POINTS  {n}  double")
        out += [f"{_g(x)} {_g(y)} 0" for x, y in g.coords]
        nc = len(g.cells)
        out.append(f"CELLS  {nc} {4 * nc}")
        out += [f"3 {a} {b} {c}" for a, b, c in g.cells]
        out.append(f"CELL_TYPES  {nc}")
        out += ["5"] * nc
        out.append(f"POINT_DATA  {n}")
        T, p, u, v = prim[:, 0], prim[:, 1], prim[:, 2], prim[:, 3]
        out += ["SCALARS pressure double 1", "LOOKUP_TABLE default"] + [_g(x, 12) for x in p]
        out += ["SCALARS temperature double 1", "LOOKUP_TABLE default"] + [_g(x, 12) for x in T]
        out += ["VECTORS velocity double"] + [f"{_g(a, 12)} {_g(b, 12)} 0" for a, b in zip(u, v)]
        if "mach" in variables:
            out += ["SCALARS mach double 1", "LOOKUP_TABLE default"]
            out += [_g(self._mach(T[i], u[i], v[i]), 12) for i in range(n)]
        if "density" in variables:
            out += ["SCALARS density double 1", "LOOKUP_TABLE default"]
            out += [_g(self._density(T[i], p[i]), 12) for i in range(n)]
        if "entropy" in variables:
            out += ["SCALARS entropy double 1", "LOOKUP_TABLE default"]
            out += [_g(self._entropy(T[i], p[i]), 12) for i in range(n)]
        if "vorticity" in variables:
            if dE is None:
                raise ValueError("vorticity needs the entropy-variable gradients dE")
            d = np.asarray(dE, np.float64).reshape(n, 5, 3)
            out += ["SCALARS vorticity double 1", "LOOKUP_TABLE default"]
            for i in range(n):                                     # src/writer.cc:238-243
                w = self.R * T[i] * (d[i, 2, 0] + v[i] * d[i, 4, 0] - d[i, 1, 1] - u[i] * d[i, 4, 1])
                out.append(_g(w, 12))
        out += ["SCALARS  dual_area  double 1", "LOOKUP_TABLE default"] + [_g(x, 12) for x in g.dcarea]
        return "\n".join(out) + "\n"

    # ------------------------------------------------------------- surfaces
    def _surface_faces(self, tag):
        return [b for b in range(self.g.n_bface) if int(self.g.bface_type[b]) == int(tag)]

    def surface_text(self, prim, tag) -> str:
        """Writer::output_surfaces: x, y, p, T, u, v, w at vertex 0 of every face of the tag."""
        prim = np.asarray(prim, np.float64).reshape(-1, 5)
        lines = []
        for b in self._surface_faces(tag):
            v0 = int(self.g.bface_vertex[b, 0])
            x, y = self.g.coords[v0]
            T, p, u, v, w = prim[v0]
            lines.append("  ".join(_g(z) for z in (x, y, p, T, u, v, w)) + "  ")
        return "".join(s + "\n" for s in lines)

    def _face_states(self, prim, b):
        v0, v1 = int(self.g.bface_vertex[b, 0]), int(self.g.bface_vertex[b, 1])
        st = []
        for slot, vv in ((0, v0), (1, v1)):
            T, p, u, v, _ = prim[vv]
            T, p, u, v = self._bc_apply(b, slot, T, p, u, v)
            st.append((T, p, u, v))
        return v0, v1, st

    def _face_center_normal(self, b, v0, v1):
        nx, ny = self.g.bface_normal[b]
        meas = math.sqrt(nx * nx + ny * ny + 0.0 * 0.0)              # src/grid_preproc.cc:321
        n = (nx * (1.0 / meas), ny * (1.0 / meas))
        (x0, y0), (x1, y1) = self.g.coords[v0], self.g.coords[v1]
        return (x0 * 0.5 + x1 * 0.5, y0 * 0.5 + y1 * 0.5), n

    def skin_friction_text(self, prim, dE, tag) -> str:
        """output_surface_sf: face centre and skin friction from the vertex gradients."""
        prim = np.asarray(prim, np.float64).reshape(-1, 5)
        d = np.asarray(dE, np.float64).reshape(-1, 5, 3)
        lines = []
        for b in self._surface_faces(tag):
            v0, v1, st = self._face_states(prim, b)
            ent = [self._prim2ent(T, p, u, v) for T, p, u, v in st]
            Tm = (st[0][0] + st[1][0]) / 2.0
            mu = self._viscosity(Tm)
            f0, f1 = 1.0 / ent[0][3], 1.0 / ent[1][3]

            def lin(a, bb, c1, c2):                                # Vector::equ, src/vec.h:254-260
                return (a[0] * c1 + bb[0] * c2, a[1] * c1 + bb[1] * c2)

            gU0 = lin(d[v0, 1], d[v0, 4], -f0, f0 * ent[0][1] / ent[0][3])
            gU1 = lin(d[v1, 1], d[v1, 4], -f1, f1 * ent[1][1] / ent[1][3])
            gU = lin(gU0, gU1, 0.5, 0.5)
            gV0 = lin(d[v0, 2], d[v0, 4], -f0, f0 * ent[0][2] / ent[0][3])
            gV1 = lin(d[v1, 2], d[v1, 4], -f1, f1 * ent[1][2] / ent[1][3])
            gV = lin(gV0, gV1, 0.5, 0.5)
            div = gU[0] + gV[1]
            sxx = 2.0 * mu * (gU[0] - (1.0 / 3.0) * div)
            syy = 2.0 * mu * (gV[1] - (1.0 / 3.0) * div)
            sxy = mu * (gU[1] + gV[0])
            (cx, cy), (nx, ny) = self._face_center_normal(b, v0, v1)
            fx = sxx * nx + sxy * ny
            fy = sxy * nx + syy * ny
            cf = fx * ny - fy * nx
            lines.append(f"{_g(cx)}  {_g(cy)}  {_g(cf)}  ")
        return "".join(s + "\n" for s in lines)

    def heat_flux_text(self, prim, dE, tag) -> str:
        """output_surface_hf: face centre and normal heat flux -k grad T . n."""
        prim = np.asarray(prim, np.float64).reshape(-1, 5)
        d = np.asarray(dE, np.float64).reshape(-1, 5, 3)
        lines = []
        for b in self._surface_faces(tag):
            v0, v1, st = self._face_states(prim, b)
            ent = [self._prim2ent(T, p, u, v) for T, p, u, v in st]
            Tm = (st[0][0] + st[1][0]) / 2.0
            mu = self._viscosity(Tm)
            k = mu * self.Cp / self.prandtl
            f0 = 1.0 / (self.R * math.pow(ent[0][3], 2.0))
            f1 = 1.0 / (self.R * math.pow(ent[1][3], 2.0))
            gT0 = (d[v0, 4, 0] * f0, d[v0, 4, 1] * f0, d[v0, 4, 2] * f0)
            gT1 = (d[v1, 4, 0] * f1, d[v1, 4, 1] * f1, d[v1, 4, 2] * f1)
            gT = tuple(a * 0.5 + c * 0.5 for a, c in zip(gT0, gT1))
            (cx, cy), (nx, ny) = self._face_center_normal(b, v0, v1)
            qn = gT[0] * nx + gT[1] * ny + gT[2] * 0.0
            qn *= -k
            lines.append(f"{_g(cx)}  {_g(cy)}  {_g(qn)}  ")
        return "".join(s + "\n" for s in lines)

    # -------------------------------------------------------------- restart
    @staticmethod
    def restart_text(prim, iteration: int, counter: int, time: float, res0: float) -> str:
        """Writer::output_restart: T, u, v, w, p per vertex (%.15e), then iteration,
        output counter, time and the first residual norm."""
        prim = np.asarray(prim, np.float64).reshape(-1, 5)
        rows = ["%.15e  %.15e  %.15e  %.15e  %.15e" % (T, u, v, w, p) for T, p, u, v, w in prim]
        return "\n".join(rows) + f"\n{int(iteration)}\n{int(counter)}\n%.15e\n%.15e\n" % (time, res0)

    # ------------------------------------------------------------- log files
    @staticmethod
    def residual_line(iteration: int, dt_global: float, elapsed: float, res_total: float,
                      steady_norms=None) -> str:
        """One residual.dat line; steady runs pass (total, mass, x, y, z momentum, energy)."""
        if steady_norms is None:
            return "%10d  %.12e  %.12e  %.12e\n" % (iteration, dt_global, elapsed, res_total)
        return ("%10d  %.4e  " % (iteration, dt_global)) + "  ".join("%.4e" % x for x in steady_norms) + "\n"

    @staticmethod
    def force_lines(iteration: int, elapsed: float, forces) -> str:
        """compute_forces' lines for one step: forces rows (inviscid x, y, viscous x, y);
        the first carries the iteration and time."""
        out = "%6d %15.6e" % (iteration, elapsed)
        for k, (fx, fy, vx, vy) in enumerate(np.asarray(forces, np.float64).reshape(-1, 4)):
            out += ("%15.6e" % fx if k == 0 else "%.6e" % fx) + "  %.6e  %.6e  %.6e\n" % (fy, vx, vy)
        return out

    @staticmethod
    def global_line(iteration: int, elapsed: float, ke: float, entropy: float) -> str:
        return f"{int(iteration)}  {_g(elapsed)}  {_g(ke)}  {_g(entropy)}\n"

    # ----------------------------------------------------- FiniteVolume::output
    def output(self, directory: str, counter: int, prim, dE=None, time=None, variables=(), surfaces=()):
        """The files FiniteVolume::output writes at output time `counter`
        (src/fv.cc:1979-2002); returns their names."""
        os.makedirs(directory, exist_ok=True)
        idx = _index(counter)
        files = {f"sol{idx}_{self.part}.vtk": self.vtk_text(prim, time, variables, dE)}
        for tag in surfaces:
            files[f"v{idx}_{self.part}_{int(tag)}.dat"] = self.surface_text(prim, tag)
        if self.ns:
            if dE is None and surfaces:
                raise ValueError("skin friction and heat flux need the entropy-variable gradients dE")
            for tag in surfaces:
                files[f"f{idx}_{self.part}_{int(tag)}.dat"] = self.skin_friction_text(prim, dE, tag)
            for tag in surfaces:
                files[f"q{idx}_{self.part}_{int(tag)}.dat"] = self.heat_flux_text(prim, dE, tag)
        for name, text in files.items():
            with open(os.path.join(directory, name), "w") as fh:
                fh.write(text)
        return list(files)
