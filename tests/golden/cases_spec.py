"""Recipes of the golden-fixture cases (shared by the generator and the tests)."""
from __future__ import annotations

import dataclasses

import numpy as np

from tensum_b200 import cases, mesh as M

WALL = {"xvelocity": 0.0, "yvelocity": 0.0, "zvelocity": 0.0}
FAR = {"temperature": 1.0 / 1.4, "xvelocity": 0.2, "yvelocity": 0.0, "zvelocity": 0.0, "pressure": 1.0 / 1.4}
PERIODIC4 = {t: ("periodic", {}) for t in (1, 2, 3, 4)}


def _sq(flux, recon, n=9, seed=3, steps=2, dump=2, ic="vortex", **kw):
    return dict(mesh="square", n=n, seed=seed, flux=flux, reconstruct=recon, ic=ic, steps=steps,
                dump_steps=dump, **kw)


def _cyl(flux, recon, model, steps=2, dump=2, bc="noslip", **kw):
    return dict(mesh="annulus", nr=6, nt=12, seed=1, flux=flux, reconstruct=recon, model=model, ic="cylinder",
                steps=steps, dump_steps=dump, wall=bc, **kw)


CASES = {
    "sq_roe_minmod": _sq("kepes_tecno_roe", "minmod"),
    "sq_rusanov_minmod": _sq("kepes_tecno_rusanov", "minmod"),
    "sq_kepec": _sq("kepec", "first"),
    "sq_kep": _sq("kep", "first"),
    "sq_roe_ec": _sq("roe_ec", "first"),
    "sq_avg": _sq("simple_avg", "first"),
    "sq_roe_first": _sq("kepes_tecno_roe", "first"),
    "sq_roe_second": _sq("kepes_tecno_roe", "second"),
    "sq_roe_vanalbada": _sq("kepes_tecno_roe", "van_albada"),
    "sq_roe_tvb": _sq("kepes_tecno_roe", "tvb_minmod", tvb_M=1.0),
    "sq_roe_eno2": _sq("kepes_tecno_roe", "eno2"),
    # unlimited MUSCL, kappa = 1/3 (src/reconstruct.cc:46-64; no parameter-file keyword)
    "sq_roe_muscl": _sq("kepes_tecno_roe", "second_muscl"),
    "sq_rusanov_muscl_long": _sq("kepes_tecno_rusanov", "second_muscl", n=17, seed=19, steps=40, dump=0),
    "cyl_ns_muscl": _cyl("kepes_tecno_roe", "second_muscl", "ns"),
    "sq_roe_evmod": _sq("kepes_tecno_roe", "minmod", ev_alpha=0.3, ev_beta=0.2),
    "sq_kh_rusanov": _sq("kepes_tecno_rusanov", "minmod", n=11, seed=5, ic="kh"),
    "vortex17_long": _sq("kepes_tecno_roe", "minmod", n=17, seed=7, steps=60, dump=0),
    "cyl_euler": _cyl("kepes_tecno_roe", "minmod", "euler"),
    "cyl_ns": _cyl("kepes_tecno_roe", "minmod", "ns"),
    "cyl_ns_rusanov_va": _cyl("kepes_tecno_rusanov", "van_albada", "ns"),
    "cyl_ns_isothermal": _cyl("kepes_tecno_roe", "minmod", "ns", bc="isothermal"),
    "cyl_slip": _cyl("kepes_tecno_roe", "minmod", "euler", bc="slip"),
    "cyl_inlet_outlet": _cyl("kepes_tecno_roe", "minmod", "euler", bc="inlet_outlet"),
    "cyl_ns_forces": _cyl("kepes_tecno_roe", "minmod", "ns", forces={"cyl": [1], "outer": [2]}),
    "cyl_slip_forces": _cyl("kepes_tecno_rusanov", "minmod", "euler", bc="slip", forces={"cyl": [1]}),
    "sq_roe_minmod_rk4": _sq("kepes_tecno_roe", "minmod", time_scheme="rk4"),
    "sq_kepec_rk4_long": _sq("kepec", "first", n=17, seed=11, steps=40, dump=0, time_scheme="rk4"),
    "cyl_ns_rk4": _cyl("kepes_tecno_roe", "minmod", "ns", time_scheme="rk4"),
    "cyl_ns_strong": _cyl("kepes_tecno_roe", "minmod", "ns", bc_scheme="strong"),
    "cyl_ns_isothermal_strong": _cyl("kepes_tecno_rusanov", "minmod", "ns", bc="isothermal", bc_scheme="strong"),
    "cyl_slip_strong": _cyl("kepes_tecno_roe", "minmod", "euler", bc="slip", bc_scheme="strong"),
    "cyl_inlet_outlet_strong": _cyl("kepec", "first", "euler", bc="inlet_outlet", bc_scheme="strong"),
    "sq_roe_liou": _sq("kepes_tecno_roe", "minmod", ic="collide", liou_fix=True, cfl=0.3),
    "sq_roe_first_liou": _sq("kepes_tecno_roe", "first", n=11, ic="collide", liou_fix=True, steps=3, dump=3, cfl=0.3),
    "sq_roe_minmod_voronoi": _sq("kepes_tecno_roe", "minmod", cell="voronoi"),
    "sq_kepec_voronoi_long": _sq("kepec", "first", n=17, seed=13, steps=40, dump=0, cell="voronoi"),
    "cyl_ns_voronoi": _cyl("kepes_tecno_roe", "minmod", "ns", cell="voronoi", forces={"cyl": [1]}),
    "sq_roe_minmod_axi": _sq("kepes_tecno_roe", "minmod", axi_shift=10.0),
    "sq_kepec_axi_long": _sq("kepec", "first", n=17, seed=17, steps=40, dump=0, axi_shift=10.0),
    "cyl_ns_axi": _cyl("kepes_tecno_roe", "minmod", "ns", axi_shift=50.0, forces={"cyl": [1]}),
    "cyl_slip_axi_voronoi": _cyl("kepes_tecno_rusanov", "minmod", "euler", bc="slip", axi_shift=50.0,
                                 cell="voronoi"),
}


def build_case(spec: dict):
    """Mesh, configuration dict and initial primitive state of one recipe."""
    if spec["mesh"] == "square":
        if spec["ic"] == "kh":
            m = M.periodic_square(spec["n"], 0.0, 1.0, 0.0, 1.0, spec["seed"])
            a, phi = cases.kh_coefficients(spec["seed"])
            prim0 = cases.kh_ic(m.coords, a, phi)
        elif spec["ic"] == "collide":
            # two streams colliding at x = 0 faster than sound: sonic points for the Liou switch
            m = cases.vortex_mesh(spec["n"], spec["seed"])
            prim0 = cases.vortex_ic(m.coords)
            prim0[:, 2] = np.where(m.coords[:, 0] < 0.0, 1.25, -1.25)
            prim0[:, 3] = 0.1 * np.sin(m.coords[:, 1])
        else:
            m = cases.vortex_mesh(spec["n"], spec["seed"])
            prim0 = cases.vortex_ic(m.coords)
        bnd = dict(PERIODIC4)
    else:
        m = M.annulus(spec["nr"], spec["nt"], 0.5, 20.0, 0.3, spec["seed"])
        prim0 = cases.cylinder_ic(m.coords)
        # perturb so that gradients and viscous terms are non-trivial
        prim0[:, 2] += 0.05 * np.sin(m.coords[:, 1])   # u (PrimVar order T, p, u, v, w)
        prim0[:, 1] *= 1.0 + 0.01 * np.cos(m.coords[:, 0])   # p
        wall = spec.get("wall", "noslip")
        if wall == "noslip":
            bnd = {1: ("noslip", WALL), 2: ("farfield", FAR)}
        elif wall == "isothermal":
            bnd = {1: ("noslip", dict(WALL, temperature=0.8)), 2: ("farfield", FAR)}
        elif wall == "slip":
            bnd = {1: ("slip", {}), 2: ("farfield", FAR)}
        else:
            bnd = {1: ("inlet", FAR), 2: ("outlet", {})}
    cfg = dict(flux=spec["flux"], reconstruct=spec["reconstruct"], boundary=bnd, final_time=100.0,
               model=spec.get("model", "euler"), mu_ref=0.002 if spec.get("model") == "ns" else 0.0,
               tvb_M=spec.get("tvb_M", 1.0), ev_alpha=spec.get("ev_alpha", 0.0), ev_beta=spec.get("ev_beta", 0.0),
               time_stamps=1, cfl=spec.get("cfl", 0.8))
    if "forces" in spec:
        cfg["forces"] = dict(spec["forces"])
    if "time_scheme" in spec:
        cfg["time_scheme"] = spec["time_scheme"]
    if spec.get("liou_fix"):
        cfg["liou_fix"] = True
    if "bc_scheme" in spec:
        cfg["bc_scheme"] = spec["bc_scheme"]
    if "cell" in spec:
        cfg["cell"] = spec["cell"]
    if spec.get("axi_shift"):
        # axisymmetric: radius = x, so the mesh is moved to x > 0 (the state moves with it)
        m = dataclasses.replace(m, coords=m.coords + np.array([spec["axi_shift"], 0.0]), name=m.name + "_axi")
        cfg["axisymmetric"] = True
    return m, cfg, prim0


# Monte Carlo case: Kelvin-Helmholtz samples whose perturbation comes from the
# rnd file through pert(4, ...) in the parameter file, run by the reference's
# own MC driver with online statistics.
MC_CASE = dict(n=17, seed=2, samples=[0, 1, 2, 3, 4], rnd_seed_base=100, flux="kepes_tecno_rusanov",
               reconstruct="minmod", final_time=0.06, time_stamps=3,
               variables=["density", "mach", "entropy", "vorticity"])
MC_EXTRAS = 1 | 2 | 4 | 8   # density, mach, entropy, vorticity


def kh_expressions(n_modes: int = 10) -> dict:
    """fparser initial condition equal to tensum_b200.cases.kh_ic_rnd."""
    terms = " + ".join(f"pert(4,x,y,{k})*sin(2*pi*{k}*x+2*pi*pert(4,x,y,{n_modes + k}))"
                       for k in range(1, n_modes + 1))
    return {"temperature": "2.5/(1+(abs(y-0.5)<0.25))", "xvelocity": "(abs(y-0.5)<0.25)-0.5",
            "yvelocity": f"0.01*({terms})", "zvelocity": "0.0", "pressure": "2.5"}


def build_mc_case(spec: dict = MC_CASE):
    """Mesh, reference configuration and per-sample random rows of the MC case."""
    m = M.periodic_square(spec["n"], 0.0, 1.0, 0.0, 1.0, spec["seed"])
    rows = {s: cases.kh_rnd_row(spec["rnd_seed_base"] + s) for s in spec["samples"]}
    cfg = dict(flux=spec["flux"], reconstruct=spec["reconstruct"], boundary=dict(PERIODIC4),
               final_time=spec["final_time"], time_stamps=spec["time_stamps"], cfl=0.8,
               samples=list(spec["samples"]), rnd_per_sample=cases.KH_RND_PER_SAMPLE, ic=kh_expressions(),
               variables=list(spec["variables"]))
    return m, cfg, rows


# Output-file cases: the reference writes its files at every output time
# (solution with derived variables, surfaces, skin friction and heat flux for
# Navier-Stokes, logs, forces, global integrals, restart).
OUTPUT_CASES = {
    "out_cyl_ns": dict(_cyl("kepes_tecno_roe", "minmod", "ns", forces={"cyl": [1]}), steps=100000,
                       final_time=0.02, time_stamps=2, surfaces=[1],
                       variables=["mach", "density", "entropy", "vorticity"]),
    "out_cyl_iso": dict(_cyl("kepes_tecno_rusanov", "minmod", "ns", bc="isothermal"), steps=100000,
                        final_time=0.01, time_stamps=1, surfaces=[1, 2], variables=["entropy"]),
    "out_sq_euler": dict(_sq("kepes_tecno_roe", "minmod"), steps=100000, final_time=0.05, time_stamps=2,
                         variables=["vorticity", "mach"]),
    # an inviscid central flux: its steps keep only V5 of the entropy variables, so
    # the written dE comes from variables formed again from the state
    "out_sq_kepec": dict(_sq("kepec", "first"), steps=100000, final_time=0.05, time_stamps=2,
                         variables=["vorticity", "mach"]),
}


def build_output_case(spec: dict):
    """Mesh, configuration (with the output keys) and initial state of an output case."""
    m, cfg, prim0 = build_case(spec)
    cfg = dict(cfg, final_time=spec["final_time"], time_stamps=spec["time_stamps"],
               variables=list(spec.get("variables", [])), surfaces=list(spec.get("surfaces", [])))
    return m, cfg, prim0


# Expression case: an initial condition using every pert type, comparisons,
# logic, if-free functions and a named constant, evaluated by the reference's
# own fparser for two samples' random numbers.
EXPR_CASE = dict(n=17, seed=4, samples=[0, 1], rnd_seed_base=300, n_rnd=8, constants={"c1": 0.0125},
                 ic={"temperature": "1.0 + 0.1*sin(2*pi*x/10)*cos(pi*y/7) + 0.02*pert(1,x,y/10+0.5,0.8)"
                                    " + 0.01*(x<0 & y>0)",
                     "xvelocity": "0.3*tanh(y) - 0.1*exp(-(x^2+y^2)/4) + 0.05*pert(3,x,(y+5)/10,0.6)"
                                  " + 0.01*((abs(x)>=2) - (abs(x)<2))",
                     "yvelocity": "0.2*pert(2,x,(x+5)/10,0.9) + 0.1*atan2(y,x+0.5)/pi + 0.01*floor(x) + c1*x",
                     "zvelocity": "0.0",
                     "pressure": "1 + 0.05*sqrt(x^2+y^2) + 0.01*pert(4,x,y,3) + 0.001*(x%3)"
                                 " + 0.02*(x>=0 | y<=-1) + 0.003*max(x,y) - 0.002*min(x,y)"
                                 " + 0.01*log(2+cosh(0.1*x)) + 0.004*!(x>1)"})


def build_expr_case(spec: dict = EXPR_CASE):
    """Mesh, reference configuration and per-sample random rows of the expression case."""
    m = cases.vortex_mesh(spec["n"], spec["seed"])
    r = np.random.default_rng(spec["rnd_seed_base"])
    rows = {s: r.uniform(0.05, 1.0, spec["n_rnd"]) for s in spec["samples"]}
    cfg = dict(flux="kepes_tecno_roe", reconstruct="minmod", boundary=dict(PERIODIC4), final_time=1.0,
               time_stamps=1, cfl=0.8, samples=list(spec["samples"]), rnd_per_sample=spec["n_rnd"],
               ic=dict(spec["ic"]), constants=dict(spec["constants"]))
    return m, cfg, rows
