"""The oracle's Monte Carlo moments reproduce the reference's MC driver.

mc_kh.npz was made by tests/golden/make_golden.py from the compiled reference:
FiniteVolume::run (src/fv.cc:2401-2492) over five Kelvin-Helmholtz samples
whose perturbation the reference evaluates from its rnd file with pert(4, ...),
online statistics of PrimVar + density, mach, entropy and vorticity at four
output instances, reduced by reduce_moments (src/reduce_moments.cc:14-221).
"""
import json

import numpy as np
import pytest

from tests.golden.cases_spec import MC_CASE, MC_EXTRAS, build_mc_case
from tests.helpers import GOLDEN
from tensum_b200 import abi, cases, preproc

import oracle as O  # noqa: E402  (tests put oracle/ on sys.path)


def _fixture():
    d = dict(np.load(f"{GOLDEN}/mc_kh.npz"))
    assert json.loads(str(d["spec"])) == MC_CASE
    return d


def _problem(mesh, cfg):
    core = {k: v for k, v in cfg.items() if k not in ("samples", "rnd_per_sample", "ic", "variables")}
    return abi.Problem(preproc.preprocess(mesh), core)


def test_product_ic_matches_reference_pert_evaluation():
    d = _fixture()
    mesh, cfg, rows = build_mc_case()
    for i, s in enumerate(MC_CASE["samples"]):
        assert np.array_equal(rows[s], d["rows"][i])
        ic = cases.kh_ic_rnd(mesh.coords, rows[s])
        # fparser and numpy evaluate sin and the mode sum independently: ulp-level agreement
        assert np.max(np.abs(ic - d["ics"][i])) <= 4e-16


def test_oracle_moments_bit_exact_with_reference_driver():
    d = _fixture()
    mesh, cfg, rows = build_mc_case()
    n_inst = len(d["time_instance"])
    n = len(MC_CASE["samples"])
    fm, sm, m2 = O.run_mc(_problem(mesh, cfg), list(d["ics"]), n_inst, MC_EXTRAS)
    for t in range(n_inst):
        O.moments_finalize(n, sm[t], m2[t])
        nvar = fm.shape[2]
        assert np.array_equal(fm[t].ravel(), d[f"m{t}_fm"]), f"mean, instance {t}"
        assert np.array_equal(sm[t].ravel(), d[f"m{t}_sm"]), f"second moment, instance {t}"
        assert np.array_equal(m2[t].ravel(), d[f"m{t}_var"]), f"variance, instance {t}"
        assert nvar == 9


def test_group_merge_matches_single_group():
    """Two MC groups merged with reduce_moments' Chan update equal one group over
    all samples up to rounding (Welford and the pairwise merge round differently)."""
    d = _fixture()
    mesh, cfg, rows = build_mc_case()
    n_inst = len(d["time_instance"])
    P = _problem(mesh, cfg)
    ics = list(d["ics"])
    a = O.run_mc(P, ics[:2], n_inst, MC_EXTRAS)
    b = O.run_mc(P, ics[2:], n_inst, MC_EXTRAS)
    for t in range(n_inst):
        fm, sm, m2 = a[0][t].copy(), a[1][t].copy(), a[2][t].copy()
        n = O.moments_merge(2, fm, sm, m2, 3, b[0][t], b[1][t], b[2][t])
        assert n == 5
        O.moments_finalize(n, sm, m2)
        # per-variable error relative to that variable's largest magnitude
        for got, key, tol in ((fm, "fm", 1e-14), (sm, "sm", 1e-14), (m2, "var", 1e-11)):
            ref = d[f"m{t}_{key}"].reshape(got.shape)
            scale = np.abs(ref).max(axis=0)
            assert np.all(np.abs(got - ref) <= tol * scale), f"{key}, instance {t}"
