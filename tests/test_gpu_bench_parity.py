"""CUDA path vs the oracle at the benchmark's own configuration.

The timed workload is the Kelvin-Helmholtz case on the seeded, jittered
1025 x 1025 periodic triangulation (1,050,625 stored vertices, 3,147,776
edges, 8,209 tiles), seed 0.  At this size the tile layout reaches its limits
(up to 235 local vertices and 491 edges of the 256 / 512 a tile holds), the
local-dt minimum runs over 8,209 blocks and the norms are formed by the last
of 8,209 blocks; the smaller parity cases reach none of these.  Every flux the
benchmark times is checked here, plus KEPES-TeCNO-Roe:

* the first-stage residual and the entropy-variable gradients against the
  oracle's compute_residual / compute_gradients (src/fv.cc:1467-1494,
  699-1059) at 1e-12 relative L2;
* five steps through tg_step -- one cold step, then four replays of the warm
  graph, the launches the benchmark times -- against the oracle's solve loop
  (src/fv.cc:2273-2305) at 1e-10 relative L2, with the clock, dt and the
  residual norm at 1e-12;
* the global entropy integral (compute_global, src/fv.cc:2175-2225) after
  every step against the oracle's at 1e-12, and the sign of its change per
  step the same as the oracle's; for the entropy-stable TeCNO fluxes it falls
  in every one of 20 steps.

A 257 x 257 Kelvin-Helmholtz run of 1000 steps (TeCNO-Roe, minmod) is checked
against the oracle at 1e-10.
"""
import numpy as np
import pytest

from tests.helpers import rel_l2
from tensum_b200 import abi, cases, gpu, preproc
import oracle as O

pytestmark = pytest.mark.gpu

BENCH_N, BENCH_SEED = 1025, 0
FLUXES = [("kep", "first"), ("kepec", "first"), ("roe_ec", "first"), ("kepes_tecno_rusanov", "minmod"),
          ("kepes_tecno_roe", "minmod")]


def _cfg(flux, recon):
    return dict(flux=flux, reconstruct=recon, boundary={t: ("periodic", {}) for t in (1, 2, 3, 4)},
                final_time=1.0e9, time_stamps=1, cfl=0.8)


@pytest.fixture(scope="module")
def kh1025():
    m = cases.kh_mesh(BENCH_N, seed=BENCH_SEED)
    a, phi = cases.kh_coefficients(BENCH_SEED)
    prim0 = cases.kh_ic(m.coords, a, phi)
    return preproc.preprocess(m), prim0


def _pair(geom, prim0, flux, recon):
    P = abi.Problem(geom, _cfg(flux, recon))
    s = gpu.Solver(P)
    s.set_state(prim0)
    o = O.Oracle(P)
    o.set_prim(prim0)
    return s, o


@pytest.mark.parametrize("flux,recon", FLUXES)
def test_kh1025_first_stage_residual_and_gradients(kh1025, flux, recon):
    geom, prim0 = kh1025
    s, o = _pair(geom, prim0, flux, recon)
    assert geom.n_vertex == 1025 * 1025
    res_o, grad_o = o.residual()
    assert rel_l2(s.residual(), res_o) <= 1e-12
    assert rel_l2(s.gradients(), grad_o) <= 1e-12


@pytest.mark.parametrize("flux,recon", FLUXES)
def test_kh1025_warm_graph_steps_and_entropy(kh1025, flux, recon):
    geom, prim0 = kh1025
    s, o = _pair(geom, prim0, flux, recon)
    ent_g = [s.global_integrals()[1]]
    ent_o = [o.global_integrals()[1]]
    assert abs(ent_g[0] - ent_o[0]) <= 1e-12 * abs(ent_o[0])
    # one cold step, then the warm graph replayed (one call of 4 steps), as timed
    for n in (1, 4):
        info = s.step(n)
        for _ in range(n):
            done, oinfo = o.step(1)
            assert done == 1
            ent_o.append(o.global_integrals()[1])
        ent_g.append(s.global_integrals()[1])
        assert abs(info[0] - oinfo[0]) <= 1e-12 * abs(oinfo[0])          # elapsed time
        assert abs(info[1] - oinfo[1]) <= 1e-12 * abs(oinfo[1])          # dt of the last step
        assert abs(info[2] - oinfo[2]) <= 1e-12 * abs(oinfo[2])          # relative residual norm
        assert int(info[3]) == int(oinfo[3])
        assert abs(ent_g[-1] - ent_o[-1]) <= 1e-12 * abs(ent_o[-1])
    assert rel_l2(s.get_state(), o.get_prim()) <= 1e-10
    # entropy production: the change over the first step and over the next four has
    # the oracle's sign wherever it is above the rounding of the integral
    dg = np.diff([ent_g[0], ent_g[1], ent_g[2]])
    do = np.diff([ent_o[0], ent_o[1], ent_o[5]])
    for a, b in zip(dg, do):
        if abs(b) > 1e-12 * abs(ent_o[0]):
            assert np.sign(a) == np.sign(b)
    if flux.startswith("kepes_tecno"):
        for _ in range(15):
            s.step(1)
            ent_g.append(s.global_integrals()[1])
        assert len(ent_g) == 18   # t = 0, after step 1, after step 5, after steps 6..20
        assert np.all(np.diff(ent_g) < 0.0), "TeCNO fluxes dissipate the mathematical entropy"


def test_kh257_tecno_roe_1000_steps_matches_oracle():
    m = cases.kh_mesh(257, seed=1)
    a, phi = cases.kh_coefficients(1)
    prim0 = cases.kh_ic(m.coords, a, phi)
    s, o = _pair(preproc.preprocess(m), prim0, "kepes_tecno_roe", "minmod")
    info = s.step(1000)
    done, oinfo = o.step(1000)
    assert done == 1000 and int(info[3]) == 1000
    assert abs(info[0] - oinfo[0]) <= 1e-12 * oinfo[0]
    assert rel_l2(s.get_state(), o.get_prim()) <= 1e-10
