"""The next step's local time step and U_old, formed by the last stage's update.

compute_dt (src/fv.cc:1499-1598) and store_conserved_old (src/fv.cc:1626-1630)
read only the state a step starts from, which the previous step's last stage
has just written; the captured step forms them there and skips the first
stage's own pass.  Same operands, same order: a run whose every step forms
them in the first stage (the state handed back in between) ends bit-identical.
"""
import numpy as np
import pytest

from tensum_b200 import abi, cases, gpu, preproc

pytestmark = pytest.mark.gpu


def _kh(flux, recon, scheme="ssprk3"):
    m = cases.kh_mesh(33, 1)
    a, phi = cases.kh_coefficients(1)
    cfg = dict(flux=flux, reconstruct=recon, boundary={t: ("periodic", {}) for t in (1, 2, 3, 4)},
               final_time=1e9, time_stamps=1, time_scheme=scheme)
    return abi.Problem(preproc.preprocess(m), cfg), cases.kh_ic(m.coords, a, phi)


def _cyl():
    m = cases.cylinder_mesh(12, 24, 1)
    cfg = cases.cylinder_config(0.2, 100.0, 1.0, 1e9, 1)
    return abi.Problem(preproc.preprocess(m), cfg), cases.cylinder_ic(m.coords, 0.2, 1.0)


@pytest.mark.parametrize("case", ["kepec", "tecno", "rk4", "cylinder"])
def test_fused_dt_is_bit_identical(case):
    if case == "cylinder":
        P, prim0 = _cyl()
    elif case == "rk4":
        P, prim0 = _kh("kepes_tecno_roe", "minmod", "rk4")
    else:
        P, prim0 = _kh(*(("kepec", "first") if case == "kepec" else ("kepes_tecno_rusanov", "minmod")))
    n = 12
    a = gpu.Solver(P)
    a.set_state(prim0)
    ia = a.step(n)
    b = gpu.Solver(P)
    b.set_state(prim0)
    for _ in range(n):
        ib = b.step(1)
        b.update_parameters(P)          # the state's dt is formed again by the next first stage
    assert np.array_equal(a.get_state(), b.get_state())
    assert ia[0] == ib[0] and ia[1] == ib[1]     # elapsed time and the last dt
