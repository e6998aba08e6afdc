"""Batched FP32 ensembles against the FP64 device solver and against themselves.

Members run in FP32, so they are compared with the FP64 path within FP32
tolerances; everything that only reorders work (launch shape, levels fused in
one launch) must be bit-identical.
"""
import numpy as np
import pytest

from tests.helpers import rel_l2
from tensum_b200 import abi, batch, cases, gpu, mc, preproc

pytestmark = pytest.mark.gpu

FLUX = ("kepes_tecno_rusanov", "minmod")


def _problem(n, seed=0, flux=FLUX, final_time=0.04, stamps=2):
    m = cases.kh_mesh(n, seed)
    cfg = dict(flux=flux[0], reconstruct=flux[1], boundary={t: ("periodic", {}) for t in (1, 2, 3, 4)},
               final_time=final_time, time_stamps=stamps, cfl=0.8)
    return m, abi.Problem(preproc.preprocess(m), cfg)


def _rows(S, base=0):
    return np.stack([cases.kh_rnd_row(base + s) for s in range(S)])


def test_device_kh_initial_condition_matches_host():
    m, P = _problem(33)
    rows = _rows(32)
    b = batch.Batch([(P, 32)])
    b.set_kh(0, rows)
    for s in (0, 7, 31):
        ref = cases.kh_ic_rnd(m.coords, rows[s])
        got = b.get_state(0, s)
        # FP32 storage of u, v, p, V1, V5; T is re-derived from p and rho
        assert np.max(np.abs(got - ref) / (np.abs(ref) + 1e-2)) <= 2e-6


@pytest.mark.parametrize("flux", [("kepes_tecno_rusanov", "minmod"), ("kepes_tecno_roe", "first"),
                                  ("kepec", "first")])
def test_fp32_members_follow_fp64_solver(flux):
    m, P = _problem(33, flux=flux)
    rows = _rows(32)
    b = batch.Batch([(P, 32)])
    b.set_kh(0, rows)
    info = b.advance(1)
    assert info[3] == 0
    s64 = gpu.Solver(P)
    for s in (0, 13):
        s64.set_state(cases.kh_ic_rnd(m.coords, rows[s]))
        s64.advance(1)
        ref = s64.get_state()
        got = b.get_state(0, s)
        assert rel_l2(got[:, :4], ref[:, :4]) <= 2e-6, s
    el, cnt, bad = b.clock(0)
    assert np.all(cnt == 2) and not bad.any()
    assert np.allclose(el, 0.02, rtol=0, atol=1e-15)


def test_launch_shapes_and_fused_levels_are_bit_identical():
    m1, P1 = _problem(17)
    m2, P2 = _problem(33, seed=1)
    r1, r2 = _rows(32), _rows(64, 100)
    ref1 = batch.Batch([(P1, 32)]); ref1.set_kh(0, r1); ref1.advance(1)
    ref2 = batch.Batch([(P2, 64)]); ref2.set_kh(0, r2); ref2.advance(1)
    n_shapes = int(ref1.query("n_shapes"))
    for shape in range(n_shapes):
        f = batch.Batch([(P1, 32), (P2, 64)])
        f.set_shape(shape)
        f.set_kh(0, r1)
        f.set_kh(1, r2)
        f.advance(1)
        for s in (0, 31):
            assert np.array_equal(f.get_state(0, s), ref1.get_state(0, s)), (shape, s)
        for s in (0, 40, 63):
            assert np.array_equal(f.get_state(1, s), ref2.get_state(0, s)), (shape, s)


def test_autotuner_restores_state_and_picks_a_shape():
    m, P = _problem(33)
    b = batch.Batch([(P, 64)])
    b.set_kh(0, _rows(64))
    before = [b.get_state(0, s) for s in (0, 63)]
    best, ms = b.tune(2)
    assert 0 <= best < len(ms) and np.all(ms > 0) and ms[best] == ms.min()
    assert int(b.query("shape")) == best
    for s, x in zip((0, 63), before):
        assert np.array_equal(b.get_state(0, s), x)
    el, cnt, _ = b.clock(0)
    assert np.all(el == 0.0) and np.all(cnt == 1)


def test_ensemble_moments_fp64_and_against_fp64_mc():
    m, P = _problem(17)
    S = 64
    rows = _rows(S)
    b = batch.Batch([(P, S)])
    b.set_kh(0, rows)
    b.advance(1)
    fm, sm, m2 = b.moments(0, extras=1 | 2 | 4)
    states = np.stack([b.get_state(0, s) for s in range(S)])        # exact FP32 states in FP64
    assert np.allclose(fm[:, :5], states.mean(axis=0), rtol=1e-13, atol=1e-15)
    var = ((states - states.mean(axis=0)) ** 2).sum(axis=0)
    assert np.all(np.abs(m2[:, :5] - var) <= 1e-10 * (np.abs(var).max(axis=0) + 1e-30))
    assert np.all(np.abs(sm[:, :5] - (states ** 2).sum(axis=0)) <= 1e-13 * np.abs(sm[:, :5]).max(axis=0))
    # the same samples as plain FP64 per-sample Monte Carlo on the device
    s64 = gpu.Solver(P)
    mc.run_group(s64, [cases.kh_ic_rnd(m.coords, r) for r in rows], 2, 1 | 2 | 4)
    f64, s64m, m264 = s64.moments_get(1)
    # FP32 members: errors relative to each field's scale, the velocity
    # components sharing the flow's velocity scale (v is small against u)
    scale = np.abs(f64).max(axis=0)
    scale[2] = scale[3] = max(scale[2], scale[3])
    scale[4] = 1.0
    assert np.all(np.abs(fm - f64) <= 2e-6 * scale)
    sd = np.sqrt(m264 / (S - 1))                                     # sample standard deviation
    sd_scale = sd.max(axis=0) + 1e-30
    got_sd = np.sqrt(np.maximum(m2, 0.0) / (S - 1))
    cols = [0, 1, 2, 3, 5, 6, 7]
    assert np.all(np.abs(got_sd - sd)[:, cols] <= 1e-3 * sd_scale[cols] + 2e-6 * scale[cols])


def test_periodic_mass_conserved_per_sample():
    m, P = _problem(33)
    b = batch.Batch([(P, 32)])
    b.set_kh(0, _rows(32))
    g = P.geom
    w = np.ones(m.n_vertex)
    for st in m.periodic_sets:
        w[st] = 1.0 / len(st)

    def mass(s):
        q = b.get_state(0, s)
        return float(np.sum(q[:, 1] / q[:, 0] * g.dcarea * w))   # rho = p / (R T), R = 1
    m0 = [mass(s) for s in (0, 5)]
    b.advance(2)
    for s, a in zip((0, 5), m0):
        assert abs(mass(s) - a) <= 2e-6 * a


def test_rejects_unsupported_setups():
    m, P = _problem(17)
    with pytest.raises(gpu.TensumError):
        batch.Batch([(P, 48)])                         # not a multiple of 32
    m2, P2 = _problem(17, flux=("kep", "first"))
    with pytest.raises(gpu.TensumError):
        batch.Batch([(P2, 32)])                        # flux without a batched kernel
    b = batch.Batch([(P, 32)])
    with pytest.raises(gpu.TensumError) as e:
        b.set_parameters(0, mu_ref=np.zeros(32))       # periodic Euler: nothing per sample
    assert abi.STATUS[e.value.status] == "TG_NOT_SUPPORTED"


def test_multilevel_moment_fields_against_fp64_ensembles():
    """Three meshes in one fused batch (the multilevel configuration at small
    sizes), advanced to one output time: each level's FP64 moment fields
    (reduce_moments' recurrence, src/reduce_moments.cc:14-221, in sample order)
    against FP64 per-sample Monte Carlo of the same samples on the device."""
    levels = [(17, 64), (33, 32), (65, 32)]
    probs, meshes, rows = [], [], []
    for i, (n, S) in enumerate(levels):
        m, P = _problem(n, seed=i, final_time=0.03, stamps=1)
        meshes.append(m); probs.append(P); rows.append(_rows(S, 1000 * i))
    b = batch.Batch([(P, S) for P, (_, S) in zip(probs, levels)])
    for i, r in enumerate(rows):
        b.set_kh(i, r)
    b.advance(1)
    for i, ((n, S), m, P) in enumerate(zip(levels, meshes, probs)):
        el, cnt, bad = b.clock(i)
        assert np.all(cnt == 2) and not bad.any() and np.allclose(el, 0.03, rtol=0, atol=1e-15)
        fm, sm, m2 = b.moments(i, extras=1 | 2 | 4)
        s64 = gpu.Solver(P)
        mc.run_group(s64, [cases.kh_ic_rnd(m.coords, r) for r in rows[i]], 2, 1 | 2 | 4)
        f64, _, m264 = s64.moments_get(1)
        scale = np.abs(f64).max(axis=0)
        scale[2] = scale[3] = max(scale[2], scale[3])
        scale[4] = 1.0
        # FP32 members, pointwise over every vertex: the finest level takes the most steps
        assert np.all(np.abs(fm - f64) <= 1e-5 * scale), n
        sd = np.sqrt(m264 / (S - 1))
        got_sd = np.sqrt(np.maximum(m2, 0.0) / (S - 1))
        cols = [0, 1, 2, 3, 5, 6, 7]
        assert np.all(np.abs(got_sd - sd)[:, cols] <= 1e-3 * (sd.max(axis=0) + 1e-30)[cols] + 1e-5 * scale[cols]), n
