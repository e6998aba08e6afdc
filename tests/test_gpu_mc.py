"""Device Monte Carlo moments against the oracle and the reference MC driver.

The samples, output times and extra variables are those of the reference MC
fixture (tests/golden/mc_kh.npz); the GPU runs each sample with tg_advance and
accumulates with tg_moments_increment, in FP64.
"""
import numpy as np
import pytest

from tests.golden.cases_spec import MC_CASE, MC_EXTRAS, build_mc_case
from tests.helpers import GOLDEN
from tensum_b200 import abi, gpu, mc, preproc

import oracle as O  # noqa: E402

pytestmark = pytest.mark.gpu

# per-variable errors relative to the variable's largest magnitude: the GPU and
# the oracle differ by flux rounding (1e-15 per stage); m2 sums squared
# deviations that are small against the mean, so it carries that relative
# difference amplified by mean/deviation
TOL = {"fm": 1e-12, "sm": 1e-12, "var": 1e-8}


def _setup():
    d = dict(np.load(f"{GOLDEN}/mc_kh.npz"))
    mesh, cfg, rows = build_mc_case()
    core = {k: v for k, v in cfg.items() if k not in ("samples", "rnd_per_sample", "ic", "variables")}
    P = abi.Problem(preproc.preprocess(mesh), core)
    return d, P


def _close(got, ref, key):
    scale = np.abs(ref).max(axis=0)
    return np.all(np.abs(got - ref) <= TOL[key] * scale)


def test_device_moments_match_oracle_and_reference_driver():
    d, P = _setup()
    n_inst = len(d["time_instance"])
    ics = list(d["ics"])
    s = gpu.Solver(P)
    n = mc.run_group(s, ics, n_inst, MC_EXTRAS)
    assert n == len(MC_CASE["samples"])
    ofm, osm, om2 = O.run_mc(P, ics, n_inst, MC_EXTRAS)
    for t in range(n_inst):
        fm, sm, m2 = s.moments_get(t)
        assert _close(fm, ofm[t], "fm") and _close(sm, osm[t], "sm") and _close(m2, om2[t], "var"), t
        s.moments_finalize(t, n)
        fm, sm, m2 = s.moments_get(t)
        for got, key in ((fm, "fm"), (sm, "sm"), (m2, "var")):
            assert _close(got, d[f"m{t}_{key}"].reshape(got.shape), key), (key, t)


def test_group_merge_host_and_device_blocks():
    import torch
    d, P = _setup()
    n_inst = len(d["time_instance"])
    ics = list(d["ics"])
    a, b, c = gpu.Solver(P), gpu.Solver(P), gpu.Solver(P)
    na = mc.run_group(a, ics[:2], n_inst, MC_EXTRAS)
    nb = mc.run_group(b, ics[2:], n_inst, MC_EXTRAS)
    mc.run_group(c, ics[:2], n_inst, MC_EXTRAS)
    nvar = a.mom_nvar
    blk = torch.empty(3 * nvar * P.geom.n_vertex, dtype=torch.float64, device="cuda")
    for t in range(n_inst):
        a.moments_merge(t, na, nb, *b.moments_get(t))
        b.moments_export(t, blk.data_ptr())
        c.moments_merge_device(t, na, nb, blk.data_ptr())
        a.moments_finalize(t, na + nb)
        c.moments_finalize(t, na + nb)
        ga, gc = a.moments_get(t), c.moments_get(t)
        for x, y in zip(ga, gc):
            assert np.array_equal(x, y)
        for got, key in zip(ga, ("fm", "sm", "var")):
            assert _close(got, d[f"m{t}_{key}"].reshape(got.shape), key), (key, t)


def test_advance_stops_at_each_output_time():
    d, P = _setup()
    tinst = d["time_instance"]
    s = gpu.Solver(P)
    s.set_state(d["ics"][0])
    for t in range(1, len(tinst)):
        info = s.advance(t)
        assert int(info[4]) == t + 1
        assert abs(info[0] - tinst[t]) <= 1e-15 * max(1.0, tinst[t])
    before = s.get_state()
    info = s.advance(len(tinst))   # past the final time: nothing left to do
    assert np.array_equal(s.get_state(), before)


def test_moment_calls_reject_bad_arguments():
    d, P = _setup()
    s = gpu.Solver(P)
    with pytest.raises(gpu.TensumError):
        s.moments_increment(0, 1)          # before tg_moments_init
    s.moments_init(2, 0)
    with pytest.raises(gpu.TensumError):
        s.moments_increment(2, 1)          # instance out of range
    with pytest.raises(gpu.TensumError):
        s.moments_increment(0, 0)          # k starts at 1
    with pytest.raises(gpu.TensumError):
        s.moments_finalize(0, 1)           # one sample has no variance
