"""Initial states and boundary values evaluated on the device from expressions.

The states the reference's fparser evaluated (tests/golden/expr_ic.npz) are
reproduced by tg_set_state_expr (FP64, device libm: a few ulp) and by
tg_batch_set_state_expr for every sample of an ensemble (FP32 records); the
per-sample boundary values of tg_batch_set_bc_expr equal the host-evaluated
table handed in through tg_batch_set_parameters.
"""
import numpy as np
import pytest

from tests.golden.cases_spec import build_expr_case
from tensum_b200 import abi, batch, cases, gpu, preproc

pytestmark = pytest.mark.gpu


def _fixture():
    import os
    from tests.helpers import GOLDEN
    return dict(np.load(os.path.join(GOLDEN, "expr_ic.npz")))


def _cfg():
    return dict(flux="kepes_tecno_roe", reconstruct="minmod", boundary={t: ("periodic", {}) for t in (1, 2, 3, 4)},
                final_time=1e9, time_stamps=1)


def test_single_solve_state_from_expressions():
    d = _fixture()
    mesh, cfg, rows = build_expr_case()
    s = gpu.Solver(abi.Problem(preproc.preprocess(mesh), _cfg()))
    fields = gpu.expr_fields(cfg["ic"], cfg["constants"])
    for k, smp in enumerate(cfg["samples"]):
        s.set_state_expr(fields, rows[smp])
        got, ref = s.get_state(), d["ics"][k]
        assert np.max(np.abs(got - ref) / (np.abs(ref) + 1e-300)) <= 1e-13
    bad = gpu.expr_fields(dict(cfg["ic"], pressure="-1 + 0*x"), cfg["constants"])
    before = s.get_state()
    with pytest.raises(gpu.TensumError):
        s.set_state_expr(bad, rows[0])
    assert np.array_equal(s.get_state(), before)      # a refused state leaves the previous one


def test_ensemble_states_from_expressions():
    d = _fixture()
    mesh, cfg, rows = build_expr_case()
    b = batch.Batch([(abi.Problem(preproc.preprocess(mesh), _cfg()), 32)])
    rr = np.stack([rows[cfg["samples"][s % 2]] for s in range(32)])
    b.set_state_expr(0, gpu.expr_fields(cfg["ic"], cfg["constants"]), rr)
    for s in (0, 1, 30, 31):
        got, ref = b.get_state(0, s), d["ics"][s % 2]
        assert np.max(np.abs(got - ref) / (np.abs(ref) + 1e-2)) <= 2e-6
    el, cnt, bad = b.clock(0)
    assert np.all(el == 0.0) and not bad.any()


def test_ensemble_boundary_values_from_expressions():
    m = cases.cylinder_mesh(10, 20, 2)
    g = preproc.preprocess(m)
    cfg = cases.cylinder_config(0.2, 100.0, 0.0, 1e9, 1)
    S = 32
    rr = np.random.default_rng(3).uniform(0.0, 1.0, (S, 2))
    far = {"temperature": "1/1.4", "xvelocity": "0.15 + 0.1*pert(4,x,y,1)",
           "yvelocity": "0.02*pert(4,x,y,2) - 0.01", "pressure": "1/1.4"}
    a = batch.Batch([(abi.Problem(g, cfg), S)])
    a.set_bc_expr(0, 2, gpu.expr_fields(far), rr)
    # the same values evaluated on the host, through the parameter table
    fields = gpu.expr_fields(far)
    vals = np.repeat(abi.bface_values(g, cfg["boundary"])[None], S, axis=0)
    for bf in np.flatnonzero(g.bface_type == 2):
        for q in range(2):
            x, y = m.coords[g.bface_vertex[bf, q]]
            for s in range(S):
                vals[s, bf, q] = [fields[0](x, y, 0, rr[s]), fields[1](x, y, 0, rr[s]), fields[2](x, y, 0, rr[s]),
                                  0.0, fields[4](x, y, 0, rr[s])]
    h = batch.Batch([(abi.Problem(g, cfg), S)])
    h.set_parameters(0, bface_values=vals)
    ic = np.stack([cases.cylinder_ic(m.coords[:1], 0.2, 0.0)[0]] * S)
    for bb in (a, h):
        bb.set_uniform(0, ic)
        bb.time_steps(5)
    for s in (0, 7, 31):
        assert np.array_equal(a.get_state(0, s), h.get_state(0, s))
    assert not np.array_equal(a.get_state(0, 0), a.get_state(0, 7))   # samples differ
    with pytest.raises(gpu.TensumError):
        a.set_bc_expr(0, 9, gpu.expr_fields(far), rr)                   # no face has tag 9
