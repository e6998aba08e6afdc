"""CUDA path vs the reference (golden fixtures) and vs the oracle (larger cases).

Tolerances (FP64): residual, gradient and residual norms per stage <= 1e-12
relative L2; dt <= 1e-13; primitive state per stage <= 1e-13 and after many
steps <= 1e-10 relative L2.  The device path differs from the reference only
through FMA contraction, summation order and last-ulp log/sqrt differences.
"""
import numpy as np
import pytest

from tests.helpers import geometry, golden_names, load_golden, rel_l2
from tensum_b200 import abi, cases, gpu, preproc
from tensum_b200 import mesh as M
import oracle as O

pytestmark = pytest.mark.gpu

TOL_RES = 1e-12
TOL_STATE_STAGE = 1e-13
TOL_STATE_LONG = 1e-10


def make_solver(mesh, cfg):
    g = geometry(mesh, cfg)
    P = abi.Problem(g, cfg)
    return gpu.Solver(P), P


@pytest.mark.parametrize("name", golden_names())
def test_stage_parity_with_reference(name):
    spec, mesh, cfg, prim0, d = load_golden(name)
    s, P = make_solver(mesh, cfg)
    s.set_state(prim0)
    if spec["dump_steps"] == 0:
        info = s.step(spec["steps"])
        assert int(info[3]) == spec["steps"]
        assert rel_l2(s.get_state(), d["prim_final"]) <= TOL_STATE_LONG
        return
    for st in range(spec["dump_steps"]):
        s.store_conserved_old()
        dtg, dt = s.compute_dt()
        assert abs(dtg - d[f"s{st}_dtg"][0]) <= 1e-13 * abs(d[f"s{st}_dtg"][0])
        assert rel_l2(dt, d[f"s{st}_dt"]) <= 1e-13
        n_rks = 4 if cfg.get("time_scheme") == "rk4" else 3
        for r in range(n_rks):
            res = s.residual()
            grad = s.gradients()
            ref_res = d[f"s{st}r{r}_res"].reshape(-1, 5)
            if r == n_rks - 1 and cfg.get("bc_scheme") == "strong":
                # the reference dump follows compute_residual_norm, which zeroed the
                # no-slip momentum residual; the norm call below zeroes ours
                res = np.where((ref_res[:, 1:4] == 0.0).all(axis=1)[:, None] & np.isin(np.arange(5), [1, 2, 3]),
                               0.0, res)
            assert rel_l2(res, ref_res) <= TOL_RES, f"residual step {st} stage {r}"
            assert rel_l2(grad, d[f"s{st}r{r}_grad"]) <= TOL_RES, f"gradient step {st} stage {r}"
            if r == n_rks - 1:
                nrm = s.residual_norm(st)
                assert rel_l2(nrm, d[f"s{st}_norm"]) <= TOL_RES
            s.update(r)
            assert rel_l2(s.get_state(), d[f"s{st}r{r}_prim"]) <= TOL_STATE_STAGE, f"state step {st} stage {r}"
        s.end_step()
        if "forces" in cfg:
            got, ref = s.forces(cfg["forces"]), d[f"s{st}_force"].reshape(-1, 4)
            # a force is a sum over a closed boundary that cancels to far below its
            # terms: the tolerance scales with the summed term magnitude max|p| sum|n|
            g = P.geom
            nrm = np.hypot(g.bface_normal[:, 0], g.bface_normal[:, 1])
            pmax = np.abs(s.get_state()[:, 1]).max()
            for f, tags in enumerate(cfg["forces"].values()):
                scale = pmax * nrm[np.isin(g.bface_type, tags)].sum()
                assert np.all(np.abs(got[f] - ref[f]) <= 1e-12 * scale), (st, f, got[f], ref[f])


def _run_pair(mesh, cfg, prim0, steps):
    s, P = make_solver(mesh, cfg)
    s.set_state(prim0)
    o = O.Oracle(P)
    o.set_prim(prim0)
    info = s.step(steps)
    done, oinfo = o.step(steps)
    assert int(info[3]) == done
    assert abs(info[0] - oinfo[0]) <= 1e-12 * max(1.0, abs(oinfo[0]))
    return s, o


KH_FLUXES = [("kep", "first"), ("kepec", "first"), ("roe_ec", "first"), ("kepes_tecno_rusanov", "minmod"),
             ("kepes_tecno_roe", "minmod")]


@pytest.mark.parametrize("flux,recon", KH_FLUXES)
def test_kh_multistep_matches_oracle(flux, recon):
    m = cases.kh_mesh(49, seed=11)
    a, phi = cases.kh_coefficients(11)
    prim0 = cases.kh_ic(m.coords, a, phi)
    cfg = dict(flux=flux, reconstruct=recon, boundary={t: ("periodic", {}) for t in (1, 2, 3, 4)},
               final_time=100.0, time_stamps=1, cfl=0.8)
    s, o = _run_pair(m, cfg, prim0, 40)
    assert rel_l2(s.get_state(), o.get_prim()) <= TOL_STATE_LONG
    ke_g, ent_g = s.global_integrals()
    ke_o, ent_o = o.global_integrals()
    assert abs(ke_g - ke_o) <= 1e-12 * abs(ke_o)
    assert abs(ent_g - ent_o) <= 1e-12 * abs(ent_o)


def test_vortex_cfg0_mesh_1000_steps_matches_oracle():
    """The 65x65 isentropic-vortex mesh, TeCNO-Roe + minmod, 1000 SSP-RK3 steps."""
    m = cases.vortex_mesh(65, seed=0)
    prim0 = cases.vortex_ic(m.coords)
    cfg = dict(flux="kepes_tecno_roe", reconstruct="minmod", boundary={t: ("periodic", {}) for t in (1, 2, 3, 4)},
               final_time=1000.0, time_stamps=1, cfl=0.8)
    s, o = _run_pair(m, cfg, prim0, 1000)
    assert rel_l2(s.get_state(), o.get_prim()) <= TOL_STATE_LONG


@pytest.mark.parametrize("recon", ["first", "second", "second_muscl", "van_albada", "tvb_minmod", "eno2"])
def test_cylinder_ns_multistep_matches_oracle(recon):
    m = M.annulus(16, 32, 0.5, 20.0, 0.05, seed=2)
    prim0 = cases.cylinder_ic(m.coords)
    prim0[:, 3] += 0.02 * np.cos(m.coords[:, 0])   # v
    cfg = dict(flux="kepes_tecno_roe", reconstruct=recon, model="ns", mu_ref=0.002, tvb_M=1.0,
               boundary={1: ("noslip", {"xvelocity": 0.0, "yvelocity": 0.0, "zvelocity": 0.0}),
                         2: ("farfield", {"temperature": 1 / 1.4, "xvelocity": 0.2, "yvelocity": 0.0,
                                          "zvelocity": 0.0, "pressure": 1 / 1.4})},
               final_time=100.0, time_stamps=1, cfl=0.8)
    s, o = _run_pair(m, cfg, prim0, 25)
    # ENO2's minabs takes the other slope at an exact tie |a| = |b| when the last
    # bit of a rounded product differs, which fused multiply-adds change: the
    # reference's own arithmetic moves by 1e-9 in one step under that change
    # (tests/test_oracle_eno2_ties.py), the device's by about 2e-7, without growth
    # (measured: at most 3e-7 over the 25 steps).  Every other reconstruction,
    # TVB minmod included, stays at 1e-15.
    tol = 1e-6 if recon == "eno2" else TOL_STATE_LONG
    assert rel_l2(s.get_state(), o.get_prim()) <= tol


def test_unsteady_clamp_hits_output_times():
    m = cases.vortex_mesh(17, seed=4)
    prim0 = cases.vortex_ic(m.coords)
    cfg = dict(flux="kepec", reconstruct="first", boundary={t: ("periodic", {}) for t in (1, 2, 3, 4)},
               final_time=0.5, time_stamps=4, cfl=0.8)
    s, o = _run_pair(m, cfg, prim0, 1000)
    info = s.step(0)
    assert info[0] == pytest.approx(0.5, abs=1e-14)
    assert rel_l2(s.get_state(), o.get_prim()) <= TOL_STATE_LONG


def test_results_are_bitwise_reproducible():
    m = cases.kh_mesh(65, seed=3)
    a, phi = cases.kh_coefficients(3)
    prim0 = cases.kh_ic(m.coords, a, phi)
    cfg = dict(flux="kepes_tecno_rusanov", reconstruct="minmod",
               boundary={t: ("periodic", {}) for t in (1, 2, 3, 4)}, final_time=100.0, time_stamps=1)
    outs = []
    for _ in range(2):
        s, _ = make_solver(m, cfg)
        s.set_state(prim0)
        s.step(20)
        outs.append(s.get_state())
    assert np.array_equal(outs[0], outs[1])


def test_periodic_residual_is_conservative():
    m = cases.kh_mesh(129, seed=5)
    a, phi = cases.kh_coefficients(5)
    prim0 = cases.kh_ic(m.coords, a, phi)
    cfg = dict(flux="kepes_tecno_roe", reconstruct="minmod",
               boundary={t: ("periodic", {}) for t in (1, 2, 3, 4)}, final_time=100.0, time_stamps=1)
    s, P = make_solver(m, cfg)
    s.set_state(prim0)
    res = s.residual()
    w = np.ones(m.n_vertex)
    for st in m.periodic_sets:
        w[st] = 1.0 / len(st)
    tot = (res * w[:, None]).sum(axis=0)
    scale = (np.abs(res) * w[:, None]).sum(axis=0)
    assert np.all(np.abs(tot[[0, 1, 2, 4]]) <= 1e-12 * scale[[0, 1, 2, 4]])


def test_tecno_entropy_decreases_and_kepec_conserves():
    m = cases.kh_mesh(65, seed=9)
    a, phi = cases.kh_coefficients(9)
    prim0 = cases.kh_ic(m.coords, a, phi)
    base = dict(boundary={t: ("periodic", {}) for t in (1, 2, 3, 4)}, final_time=100.0, time_stamps=1)
    s, _ = make_solver(m, dict(base, flux="kepes_tecno_rusanov", reconstruct="minmod"))
    s.set_state(prim0)
    ent = [s.global_integrals()[1]]
    for _ in range(10):
        s.step(1)
        ent.append(s.global_integrals()[1])
    assert np.all(np.diff(ent) < 0.0)  # mathematical entropy -rho s/(gamma-1) is dissipated
    s2, _ = make_solver(m, dict(base, flux="kepec", reconstruct="first"))
    s2.set_state(prim0)
    e0 = s2.global_integrals()[1]
    s2.step(10)
    e1 = s2.global_integrals()[1]
    assert abs(e1 - e0) <= 1e-6 * abs(e0)  # entropy conservative up to time-integration error
