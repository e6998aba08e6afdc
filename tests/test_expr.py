"""Parameter-file expressions compiled by the library and evaluated on the host.

The reference evaluates its initial and boundary conditions with fparser
(src/fparser.h:20-36) and pert() (src/perturb.cc:16-208); the fixtures hold
states the reference itself evaluated from its parameter file, so the
library's compiler and evaluator (the same code the device kernels run) are
pinned against them.  Differences are the last-ulp effects of fparser's
parse-time rewrites; the bound is stated below.
"""
import json
import os

import numpy as np
import pytest

from tests.helpers import GOLDEN
from tests.golden.cases_spec import EXPR_CASE, build_expr_case, build_mc_case, kh_expressions
from tensum_b200 import gpu

REL = 1e-14


def _eval_state(fields, coords, row):
    out = np.zeros((coords.shape[0], 5))
    cols = (0, 2, 3, 4, 1)   # fields T, u, v, w, p -> PrimVar memory order T, p, u, v, w
    for c, f in enumerate(fields):
        if f is None:
            continue
        out[:, cols[c]] = [f(x, y, 0.0, row) for x, y in coords]
    return out


def _rel(a, b):
    return np.max(np.abs(a - b) / (np.abs(b) + 1e-300))


def test_grammar_and_fparser_semantics():
    E = gpu.Expr
    assert E("-2^2")(0, 0) == -4.0 and E("2^3^2")(0, 0) == 512.0 and E("2^-1")(0, 0) == 0.5
    assert E("1+2*3-4/2")(0, 0) == 5.0 and E("7%3")(0, 0) == 1.0
    # comparisons carry fparser's 1e-12 tolerance; truth is |v| >= 0.5
    assert E("0.25 < 0.25 + 5e-13")(0, 0) == 0.0 and E("0.25 = 0.25 + 5e-13")(0, 0) == 1.0
    assert E("0.4 & 1")(0, 0) == 0.0 and E("0.6 & 1")(0, 0) == 1.0 and E("!0.4")(0, 0) == 1.0
    assert E("if(x < 0, 1, 2)")(-1, 0) == 1.0 and E("if(x < 0, 1, 2)")(1, 0) == 2.0
    assert E("a*x + b", {"a": 2.0, "b": 1.0})(3, 0) == 7.0 and E("pi")(0, 0) == np.pi
    assert E("pert(4, x, y, 2)")(0, 0, 0, [0.5, 0.7]) == 0.7
    for bad in ("sin(", "foo(x)", "q + 1", "pert(1, x)", "1 +"):
        with pytest.raises(gpu.TensumError):
            E(bad)
    with pytest.raises(gpu.TensumError):
        E("pert(4, x, y, 5)")(0, 0, 0, [0.1, 0.2])      # no fifth random number


def test_expression_case_matches_the_reference_fparser():
    d = dict(np.load(os.path.join(GOLDEN, "expr_ic.npz")))
    assert json.loads(str(d["spec"])) == EXPR_CASE
    mesh, cfg, rows = build_expr_case()
    fields = gpu.expr_fields(cfg["ic"], cfg["constants"])
    for k, s in enumerate(cfg["samples"]):
        assert np.array_equal(d["rows"][k], rows[s])
        got = _eval_state(fields, mesh.coords, rows[s])
        assert _rel(got, d["ics"][k]) <= REL, _rel(got, d["ics"][k])


def test_kelvin_helmholtz_pert_expressions_match_the_reference():
    d = dict(np.load(os.path.join(GOLDEN, "mc_kh.npz")))
    mesh, cfg, rows = build_mc_case()
    fields = gpu.expr_fields(kh_expressions())
    for k, s in enumerate(cfg["samples"][:2]):
        got = _eval_state(fields, mesh.coords, rows[s])
        assert _rel(got, d["ics"][k]) <= REL
