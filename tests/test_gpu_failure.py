"""Failure detection without a GPU fault: states that blow up are flagged.

The failure is made on the host (a time step far beyond the stability limit);
the update kernels flag non-finite values or p <= 0 / rho <= 0 and the calls
return TG_BAD_STATE, with the context still usable afterwards.
"""
import numpy as np
import pytest

from tensum_b200 import abi, batch, cases, gpu, preproc

pytestmark = pytest.mark.gpu


def _problem(cfl, final_time=100.0, flux="kepec", recon="first"):
    m = cases.kh_mesh(33, 0)
    cfg = dict(flux=flux, reconstruct=recon, boundary={t: ("periodic", {}) for t in (1, 2, 3, 4)},
               final_time=final_time, time_stamps=1, cfl=cfl)
    return m, abi.Problem(preproc.preprocess(m), cfg)


def test_unstable_step_is_flagged_and_context_survives():
    m, P = _problem(cfl=60.0)
    s = gpu.Solver(P)
    a, phi = cases.kh_coefficients(0)
    s.set_state(cases.kh_ic(m.coords, a, phi))
    with pytest.raises(gpu.TensumError) as e:
        for _ in range(50):
            s.step(1)
    assert abi.STATUS[e.value.status] == "TG_BAD_STATE"
    # the same handle (and context) runs a sane state again
    m2, P2 = _problem(cfl=0.8)
    s2 = gpu.Solver(P2)
    s2.set_state(cases.kh_ic(m2.coords, a, phi))
    s2.step(5)
    assert np.all(np.isfinite(s2.get_state()))


def test_ensemble_flags_only_the_failing_samples():
    m, P = _problem(cfl=0.8, final_time=0.05, flux="kepes_tecno_rusanov", recon="minmod")
    b = batch.Batch([(P, 32)])
    rows = np.stack([cases.kh_rnd_row(s) for s in range(32)])
    b.set_kh(0, rows)
    bad = cases.kh_ic_rnd(m.coords, rows[5])
    bad[:, 3] *= 1.0e4          # sample 5: a velocity field far beyond anything the CFL step tolerates
    bad[:, 2] += 300.0
    b.set_state(0, 5, bad)
    with pytest.raises(gpu.TensumError) as e:
        b.advance(1)
    assert abi.STATUS[e.value.status] == "TG_BAD_STATE"
    el, cnt, flags = b.clock(0)
    assert flags[5] == 1 and flags.sum() == 1
    assert np.all(cnt[np.arange(32) != 5] == 2)
