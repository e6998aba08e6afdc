"""Per-sample material constants and boundary values on one handle.

A Monte Carlo sample of the cylinder changes the inflow Mach number and angle
(far-field values, src/bc.h:568-654) and the viscosity (Re); the mesh, the
schemes and the boundary kinds stay.  tg_update_parameters must leave the
handle in the state a fresh tg_create with the sample's parameters would give:
the same bits after the same steps, forces included (src/force.cc:116-219).
"""
import numpy as np
import pytest

from tensum_b200 import abi, cases, gpu, preproc, qoi

pytestmark = pytest.mark.gpu


def _run(s, m, mach, angle, n):
    s.set_state(cases.cylinder_ic(m.coords, mach, angle))
    f = []
    for _ in range(n):
        s.step(5)
        f.append(s.forces({"cylinder": [1]})[0])
    return s.get_state(), np.array(f)


@pytest.mark.parametrize("recon", ["first", "minmod"])
def test_updated_handle_matches_fresh_handle(recon):
    m = cases.cylinder_mesh(16, 32, 3)
    g = preproc.preprocess(m)
    a = (0.2, 100.0, 1.0)
    b = (0.16, 85.0, -1.7)
    s = gpu.Solver(abi.Problem(g, cases.cylinder_config(*a, 1e9, 1, recon=recon)))
    _run(s, m, a[0], a[2], 2)   # the old parameters have run and the step graph exists
    s.update_parameters(abi.Problem(g, cases.cylinder_config(*b, 1e9, 1, recon=recon)))
    got, fgot = _run(s, m, b[0], b[2], 4)
    ref = gpu.Solver(abi.Problem(g, cases.cylinder_config(*b, 1e9, 1, recon=recon)))
    want, fwant = _run(ref, m, b[0], b[2], 4)
    assert np.array_equal(got, want)
    assert np.array_equal(fgot, fwant)
    cd, cl = qoi.force_coefficients(fgot, b[0], b[2])
    assert np.all(np.isfinite(cd)) and np.all(np.isfinite(cl))


def test_update_parameters_refuses_other_schemes():
    m = cases.cylinder_mesh(8, 16, 0)
    g = preproc.preprocess(m)
    s = gpu.Solver(abi.Problem(g, cases.cylinder_config(0.2, 100.0, 0.0, 1e9, 1)))
    with pytest.raises(gpu.TensumError) as e:
        s.update_parameters(abi.Problem(g, cases.cylinder_config(0.2, 100.0, 0.0, 1e9, 1, flux="kepec")))
    assert abi.STATUS[e.value.status] == "TG_NOT_SUPPORTED"
