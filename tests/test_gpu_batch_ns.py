"""Batched FP32 Navier-Stokes ensembles on the cylinder O-mesh.

Every sample has its own free stream (Mach, inflow angle: far-field values,
src/bc.h:568-654) and viscosity (Re); the walls are adiabatic no-slip.  The
members run in FP32 and follow the FP64 single solve of the same sample
(weak boundary fluxes src/fv.cc:1100-1188, viscous units src/fv.cc:1197-1320,
forces src/force.cc:116-219) within FP32 tolerances; reordering work (launch
shape) must not change a bit.
"""
import numpy as np
import pytest

from tests.helpers import rel_l2
from tensum_b200 import abi, batch, cases, gpu, preproc

pytestmark = pytest.mark.gpu

FORCES = {"cylinder": [1]}


def _params(S, seed=0):
    r = np.random.default_rng(seed)
    return np.stack([r.uniform(0.15, 0.25, S), r.uniform(80.0, 120.0, S), r.uniform(-2.0, 2.0, S)], axis=1)


def _setup(flux, recon, S=32, n_r=16, n_t=32, final_time=0.03, stamps=1, seed=0):
    m = cases.cylinder_mesh(n_r, n_t, seed)
    g = preproc.preprocess(m)
    prm = _params(S, seed)
    cfgs = [cases.cylinder_config(*p, final_time, stamps, flux=flux, recon=recon) for p in prm]
    P = abi.Problem(g, cfgs[0])
    b = batch.Batch([(P, S)])
    b.set_parameters(0, mu_ref=[c["mu_ref"] for c in cfgs],
                     bface_values=np.stack([abi.bface_values(g, c["boundary"]) for c in cfgs]))
    b.set_uniform(0, np.stack([cases.cylinder_ic(m.coords[:1], p[0], p[2])[0] for p in prm]))
    return m, g, prm, cfgs, b


@pytest.mark.parametrize("flux,recon", [("kepes_tecno_roe", "minmod"), ("kepes_tecno_rusanov", "first"),
                                        ("kepec", "first")])
def test_fp32_members_follow_fp64_solver(flux, recon):
    m, g, prm, cfgs, b = _setup(flux, recon)
    info = b.advance(1)
    assert info[3] == 0
    el, cnt, bad = b.clock(0)
    assert not bad.any() and np.all(cnt == 2)
    assert np.allclose(el, 0.03, rtol=0, atol=1e-15)
    fb = b.forces(0, FORCES)
    errs, ferrs = [], []
    s64 = None
    for s in (0, 5, 31):
        P = abi.Problem(g, cfgs[s])
        if s64 is None:
            s64 = gpu.Solver(P)
        else:
            s64.update_parameters(P)
        s64.set_state(cases.cylinder_ic(m.coords, prm[s][0], prm[s][2]))
        s64.advance(1)
        ref = s64.get_state()
        got = b.get_state(0, s)
        errs.append(rel_l2(got[:, :4], ref[:, :4]))
        f64 = s64.forces(FORCES)[0]
        scale = np.max(np.abs(f64[:2])) + 1e-30
        ferrs.append(np.max(np.abs(fb[s, 0] - f64)) / scale)
    print("fp32 vs fp64 state rel L2", errs, "forces", ferrs)
    assert max(errs) <= 2e-5
    assert max(ferrs) <= 2e-3


def test_launch_shapes_are_bit_identical():
    states = []
    forces = []
    for shape in range(4):
        m, g, prm, cfgs, b = _setup("kepes_tecno_roe", "minmod", final_time=0.01)
        b.set_shape(shape)
        b.advance(1)
        states.append(np.stack([b.get_state(0, s) for s in (0, 17, 31)]))
        forces.append(b.forces(0, FORCES))
    for x in states[1:]:
        assert np.array_equal(x, states[0])
    for x in forces[1:]:
        assert np.array_equal(x, forces[0])


def test_sample_parameters_are_independent():
    """Two samples given the same parameters end bitwise equal; a third differs."""
    m = cases.cylinder_mesh(12, 24, 1)
    g = preproc.preprocess(m)
    cfg_a = cases.cylinder_config(0.2, 100.0, 1.0, 0.01, 1)
    cfg_b = cases.cylinder_config(0.17, 90.0, -1.0, 0.01, 1)
    b = batch.Batch([(abi.Problem(g, cfg_a), 32)])
    cfgs = [cfg_b if s in (3, 30) else cfg_a for s in range(32)]
    b.set_parameters(0, mu_ref=[c["mu_ref"] for c in cfgs],
                     bface_values=np.stack([abi.bface_values(g, c["boundary"]) for c in cfgs]))
    ic = [cases.cylinder_ic(m.coords[:1], 0.17, -1.0)[0] if s in (3, 30) else cases.cylinder_ic(m.coords[:1], 0.2, 1.0)[0]
          for s in range(32)]
    b.set_uniform(0, np.stack(ic))
    b.advance(1)
    assert np.array_equal(b.get_state(0, 3), b.get_state(0, 30))
    assert np.array_equal(b.get_state(0, 0), b.get_state(0, 31))
    assert not np.array_equal(b.get_state(0, 0), b.get_state(0, 3))
    f = b.forces(0, FORCES)
    assert np.array_equal(f[3], f[30]) and np.all(np.isfinite(f))


def test_unsupported_options_are_refused():
    m = cases.cylinder_mesh(8, 16, 0)
    g = preproc.preprocess(m)
    for extra in ({"bc_scheme": "strong"}, {"liou_fix": True}):
        cfg = dict(cases.cylinder_config(0.2, 100.0, 0.0, 0.01, 1), **extra)
        with pytest.raises(gpu.TensumError) as e:
            batch.Batch([(abi.Problem(g, cfg), 32)])
        assert abi.STATUS[e.value.status] == "TG_NOT_SUPPORTED"
