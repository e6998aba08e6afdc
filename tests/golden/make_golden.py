"""Generate golden fixtures by running the TENSUM reference itself.

Needs the reference tree and a built oracle/_ref/tensum_harness (``make -C
oracle ref``); run from the repository root:

    python tests/golden/make_golden.py

Every fixture records the case recipe (mesh generator + seed, boundary and
scheme configuration), the initial state handed to the reference, and the
reference's per-stage arrays dumped at full precision.  Tests rebuild the mesh
from the recipe (the generators are deterministic) and compare against these
arrays, so the checks run on machines without the reference.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from tests.golden.cases_spec import build_mc_case, MC_CASE, CASES, build_case, EXPR_CASE, build_expr_case  # noqa: E402
import ref_runner  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def main():
    if not ref_runner.harness_available():
        raise SystemExit("oracle/_ref/tensum_harness missing: run `make -C oracle ref` first")
    only = set(sys.argv[1:])
    for name, spec in CASES.items():
        if only and name not in only:
            continue
        mesh, cfg, prim0 = build_case(spec)
        d = ref_runner.run_case(mesh, cfg, prim0, spec["steps"], spec["dump_steps"])
        keep = {k: v for k, v in d.items() if k not in ("wall_s", "step_s")}   # timings are not fixtures
        keep["prim_in"] = prim0.ravel()
        np.savez_compressed(os.path.join(OUT, f"{name}.npz"), spec=np.array(json.dumps(spec)), **keep)
        print(name, "vertices", mesh.n_vertex, "records", len(keep))
    if not only or "mc_kh" in only:
        make_mc()
    if not only or "expr_ic" in only:
        make_expr()


def make_expr():
    """expr_ic.npz: initial states the reference evaluates with its fparser from
    the expression case's parameter file, one per sample's random numbers."""
    mesh, cfg, rows = build_expr_case()
    ics = []
    for s in cfg["samples"]:
        one = ref_runner.run_case(mesh, dict(cfg, samples=[s]), None, 0, 0, rnd_rows=rows)
        ics.append(one["prim0"].reshape(-1, 5))
    np.savez_compressed(os.path.join(OUT, "expr_ic.npz"), spec=np.array(json.dumps(EXPR_CASE)), ics=np.stack(ics),
                        rows=np.stack([rows[s] for s in cfg["samples"]]))
    print("expr_ic vertices", mesh.n_vertex, "samples", len(ics))


def make_mc():
    """mc_kh.npz: the reference MC driver's reduced moments and each sample's
    initial state as the reference evaluates it (fparser + pert from the rnd file)."""
    mesh, cfg, rows = build_mc_case()
    d = ref_runner.run_mc(mesh, cfg, rows)
    ics = []
    for s in cfg["samples"]:
        one = ref_runner.run_case(mesh, dict(cfg, samples=[s]), None, 0, 0, rnd_rows=rows)
        ics.append(one["prim0"].reshape(-1, 5))
    keep = {k: v for k, v in d.items() if k.startswith("m") or k in ("time_instance", "n_samples")}
    keep["ics"] = np.stack(ics)
    keep["rows"] = np.stack([rows[s] for s in cfg["samples"]])
    np.savez_compressed(os.path.join(OUT, "mc_kh.npz"), spec=np.array(json.dumps(MC_CASE)), **keep)
    print("mc_kh vertices", mesh.n_vertex, "instances", len(d["time_instance"]), "samples", int(d["n_samples"][0]))


if __name__ == "__main__":
    main()
