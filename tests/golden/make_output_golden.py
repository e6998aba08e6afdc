"""Golden output files: the reference writes its own solution, surface, log,
force, global and restart files, and the exact state and gradients each
output time wrote are kept next to them.

Needs the reference tree and a built oracle/_ref/tensum_harness (``make -C
oracle ref``); run from the repository root:

    python tests/golden/make_output_golden.py [case ...]

Tests regenerate every file with tensum_b200.writer from the kept arrays and
compare the text byte for byte, and compare device snapshots with the arrays.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from tests.golden.cases_spec import OUTPUT_CASES, build_output_case  # noqa: E402
import ref_runner  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def main():
    if not ref_runner.harness_available():
        raise SystemExit("oracle/_ref/tensum_harness missing: run `make -C oracle ref` first")
    names = sys.argv[1:] or list(OUTPUT_CASES)
    for name in names:
        spec = OUTPUT_CASES[name]
        mesh, cfg, prim0 = build_output_case(spec)
        d, texts = ref_runner.run_files(mesh, cfg, prim0, spec["steps"])
        keep = {k: v for k, v in d.items() if k.startswith("o") or k in (
            "prim_final", "restart_res0", "restart_counter", "iters", "elapsed", "steps_run")}
        keep["prim_in"] = prim0.ravel()
        np.savez_compressed(os.path.join(OUT, f"{name}.npz"), spec=np.array(json.dumps(spec)),
                            files=np.array(json.dumps(texts)), **keep)
        print(name, sorted(texts))


if __name__ == "__main__":
    main()
