"""Synthetic workloads: meshes, initial conditions and boundary conditions.

Each case is a seeded stand-in for one of the reference's benchmark setups;
initial conditions are returned in the reference's PrimVar order
(T, p, u, v, w) per vertex (src/primvar.h:17-18), i.e. exactly the array a
reference caller hands to ``tg_set_state``.
"""
from __future__ import annotations

import numpy as np

from . import mesh as _mesh

GAMMA = 1.4


def vortex_mesh(n: int = 65, seed: int = 0) -> _mesh.TriMesh:
    """Isentropic-vortex mesh: [-5,5]^2 periodic, n x n vertices."""
    return _mesh.periodic_square(n, -5.0, 5.0, -5.0, 5.0, seed, name=f"vortex{n}")


def vortex_ic(coords: np.ndarray, beta: float = 5.0, gamma: float = GAMMA,
              u_inf: float = 1.0, v_inf: float = 1.0, gas_const: float = 1.0) -> np.ndarray:
    """Isentropic vortex (strength beta) centred at the origin in a (1,1,1,1) stream."""
    x, y = coords[:, 0], coords[:, 1]
    r2 = x * x + y * y
    T = 1.0 - (gamma - 1.0) * beta * beta / (8.0 * gamma * np.pi * np.pi) * np.exp(1.0 - r2)
    e = np.exp(0.5 * (1.0 - r2))
    u = u_inf - beta / (2.0 * np.pi) * y * e
    v = v_inf + beta / (2.0 * np.pi) * x * e
    p = T ** (gamma / (gamma - 1.0))
    rho = p / (gas_const * T)
    T = p / (gas_const * rho)
    return np.stack([T, p, u, v, np.zeros_like(T)], axis=1)


def kh_mesh(n: int = 1025, seed: int = 0) -> _mesh.TriMesh:
    """Kelvin-Helmholtz mesh: [0,1]^2 periodic, n x n vertices."""
    return _mesh.periodic_square(n, 0.0, 1.0, 0.0, 1.0, seed, name=f"kh{n}")


def kh_coefficients(seed: int, n_modes: int = 10):
    """Perturbation amplitudes a_k ~ U[0,1] and phases phi_k ~ U[0, 2 pi)."""
    rng = np.random.default_rng(seed)
    a = rng.uniform(0.0, 1.0, n_modes)
    phi = rng.uniform(0.0, 2.0 * np.pi, n_modes)
    return a, phi


KH_RND_PER_SAMPLE = 20


def kh_rnd_row(seed: int, n_modes: int = 10) -> np.ndarray:
    """One sample's random numbers in the layout of the reference's rnd file
    (src/fv.cc:502-551): r_1..r_M are the amplitudes a_k ~ U[0,1] and
    r_{M+1}..r_{2M} the phases as fractions of a turn, phi_k = 2 pi r_{M+k}."""
    rng = np.random.default_rng(seed)
    return rng.uniform(0.0, 1.0, 2 * n_modes)


def kh_expressions(n_modes: int = 10) -> dict:
    """The Kelvin-Helmholtz initial condition as the parameter file's
    expressions: the layer and the seeded perturbation through pert(4, ...)
    over the sample's rnd-file row (src/perturb.cc:196-208), equal to
    kh_ic_rnd."""
    terms = " + ".join(f"pert(4,x,y,{k})*sin(2*pi*{k}*x+2*pi*pert(4,x,y,{n_modes + k}))"
                       for k in range(1, n_modes + 1))
    return {"temperature": "2.5/(1+(abs(y-0.5)<0.25))", "xvelocity": "(abs(y-0.5)<0.25)-0.5",
            "yvelocity": f"0.01*({terms})", "zvelocity": "0.0", "pressure": "2.5"}


def kh_ic_rnd(coords: np.ndarray, row: np.ndarray, gas_const: float = 1.0) -> np.ndarray:
    """The Kelvin-Helmholtz initial state of one Monte Carlo sample from its
    random-number row.  It is the value of the parameter-file initial condition

        yvelocity  0.01*(pert(4,x,y,1)*sin(2*pi*1*x+2*pi*pert(4,x,y,M+1)) + ...
                         + pert(4,x,y,M)*sin(2*pi*M*x+2*pi*pert(4,x,y,2M)))

    (pert type 4 returns r_id, src/perturb.cc:196-208) with the shear layer of
    kh_ic, summed over the modes in order."""
    m = row.size // 2
    x, y = coords[:, 0], coords[:, 1]
    s = np.zeros_like(x)
    for k in range(1, m + 1):
        s = s + row[k - 1] * np.sin(2.0 * np.pi * k * x + 2.0 * np.pi * row[m + k - 1])
    inside = np.abs(y - 0.5) < 0.25
    rho = np.where(inside, 2.0, 1.0)
    p = np.full_like(x, 2.5)
    return np.stack([p / (gas_const * rho), p, np.where(inside, 0.5, -0.5), 0.01 * s, np.zeros_like(x)], axis=1)


def kh_ic(coords: np.ndarray, a: np.ndarray, phi: np.ndarray, gas_const: float = 1.0) -> np.ndarray:
    """Kelvin-Helmholtz shear layer with a multimodal vertical-velocity perturbation."""
    x, y = coords[:, 0], coords[:, 1]
    inside = np.abs(y - 0.5) < 0.25
    rho = np.where(inside, 2.0, 1.0)
    u = np.where(inside, 0.5, -0.5)
    k = np.arange(1, a.size + 1)
    v = 0.01 * np.sum(a[None, :] * np.sin(2.0 * np.pi * k[None, :] * x[:, None] + phi[None, :]), axis=1)
    p = np.full_like(x, 2.5)
    T = p / (gas_const * rho)
    return np.stack([T, p, u, v, np.zeros_like(T)], axis=1)


def cylinder_mesh(n_r: int = 256, n_t: int = 512, seed: int = 0) -> _mesh.TriMesh:
    """O-mesh around a unit-diameter cylinder out to radius 20."""
    return _mesh.annulus(n_r, n_t, 0.5, 20.0, 2.0e-3, seed, name=f"cyl{n_r}x{n_t}")


def cylinder_freestream(mach: float = 0.2, angle_deg: float = 0.0, gamma: float = GAMMA,
                        gas_const: float = 1.0):
    """Free stream with rho = 1, p = 1/gamma (sound speed 1), speed = Mach."""
    p = 1.0 / gamma
    rho = 1.0
    T = p / (gas_const * rho)
    th = np.deg2rad(angle_deg)
    return T, mach * np.cos(th), mach * np.sin(th), p


def cylinder_ic(coords: np.ndarray, mach: float = 0.2, angle_deg: float = 0.0) -> np.ndarray:
    T, u, v, p = cylinder_freestream(mach, angle_deg)
    n = coords.shape[0]
    return np.stack([np.full(n, T), np.full(n, p), np.full(n, u), np.full(n, v), np.zeros(n)], axis=1)


def cylinder_config(mach: float, reynolds: float, angle_deg: float, final_time: float, time_stamps: int,
                    flux: str = "kepes_tecno_roe", recon: str = "minmod", cfl: float = 0.8) -> dict:
    """Navier-Stokes flow past the cylinder: adiabatic no-slip wall (tag 1),
    characteristic far field at the free stream (tag 2), Pr 0.72, and the force
    on the wall as the integrals section would define it."""
    T, u, v, p = cylinder_freestream(mach, angle_deg)
    far = {"temperature": T, "xvelocity": u, "yvelocity": v, "zvelocity": 0.0, "pressure": p}
    wall = {"xvelocity": 0.0, "yvelocity": 0.0, "zvelocity": 0.0}
    return dict(flux=flux, reconstruct=recon, model="ns", mu_ref=cylinder_viscosity(mach, reynolds), prandtl=0.72,
                boundary={1: ("noslip", wall), 2: ("farfield", far)}, final_time=final_time,
                time_stamps=time_stamps, cfl=cfl, forces={"cylinder": [1]})


def cylinder_viscosity(mach: float = 0.2, reynolds: float = 100.0, diameter: float = 1.0) -> float:
    """Constant viscosity giving Re = rho U D / mu with rho = 1."""
    return mach * diameter / reynolds
