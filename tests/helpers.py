"""Helpers shared by the tests: golden fixtures and error metrics."""
from __future__ import annotations

import glob
import json
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def golden_names():
    """Single-solve fixtures (the Monte Carlo fixtures mc_*.npz, the output-file
    fixtures out_*.npz and the expression fixture expr_*.npz have their own tests)."""
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz"))
                  if not os.path.basename(p).startswith(("mc_", "out_", "expr_")))


def load_golden(name):
    from tests.golden.cases_spec import build_case
    d = dict(np.load(os.path.join(GOLDEN, f"{name}.npz")))
    spec = json.loads(str(d.pop("spec")))
    mesh, cfg, prim0 = build_case(spec)
    assert np.array_equal(prim0.ravel(), d["prim_in"]), "case recipe no longer reproduces the fixture input"
    return spec, mesh, cfg, prim0, d


def rel_l2(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    n = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / n) if n > 0 else float(np.linalg.norm(a - b))


def geometry(mesh, cfg):
    """The preprocessed geometry a fixture's configuration asks for (dual cell type, axisymmetry)."""
    from tensum_b200 import preproc
    return preproc.preprocess(mesh, cell=cfg.get("cell", "median"), axisymmetric=cfg.get("axisymmetric", False))
