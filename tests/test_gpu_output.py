"""Asynchronous output snapshots against the reference's own output times.

At every output time the reference writes primitive and dE (src/fv.cc:
1979-2002); the device snapshot taken by tg_output_begin, with steps of the
next interval enqueued before tg_output_wait, must hold the same arrays
(FP64 tolerances), and the files written from it must match the reference's
line structure and numbers.
"""
import json
import os
import re

import numpy as np
import pytest

from tests.helpers import GOLDEN
from tests.golden.cases_spec import OUTPUT_CASES, build_output_case
from tensum_b200 import abi, gpu, preproc, writer

pytestmark = pytest.mark.gpu


def _load(name):
    d = dict(np.load(os.path.join(GOLDEN, f"{name}.npz")))
    spec = json.loads(str(d.pop("spec")))
    files = json.loads(str(d.pop("files")))
    mesh, cfg, prim0 = build_output_case(spec)
    return spec, cfg, mesh, prim0, d, files


def _numbers(text):
    return np.array([float(x) for x in re.findall(r"[-+]?\d*\.?\d+(?:[eE][-+]?\d+)?|nan|inf", text)])


@pytest.mark.parametrize("name", sorted(OUTPUT_CASES))
def test_snapshots_match_reference_outputs(name):
    spec, cfg, mesh, prim0, d, files = _load(name)
    g = preproc.preprocess(mesh)
    s = gpu.Solver(abi.Problem(g, cfg))
    s.set_state(prim0)
    w = writer.Writer(g, cfg)
    ns_forces = cfg.get("model") == "ns" and "forces" in cfg
    prim, grad = s.output_buffers()
    n_out = spec["time_stamps"]
    for k in range(n_out + 1):
        if k > 0:
            s.advance(k)
        grad_state = s.GRAD_LAST_STAGE
        if ns_forces and k > 0:
            s.forces(cfg["forces"])        # compute_forces recomputes dE of the current state first
            grad_state = s.GRAD_CURRENT
        s.output_begin(prim, grad, grad_state)
        if k < n_out:
            s.step(3)                      # the next interval's steps overlap the copy
        s.output_wait()
        ref_p, ref_g = d[f"o{k}_prim"].reshape(-1, 5), d[f"o{k}_grad"].reshape(-1, 5, 3)
        scale = np.max(np.abs(ref_p), axis=0) + 1e-300
        assert np.max(np.abs(prim - ref_p) / scale) <= 1e-10, k
        gs = np.max(np.abs(ref_g)) + 1e-300
        assert np.max(np.abs(grad - ref_g)) <= 1e-8 * gs, k
        if k < n_out:
            s.set_state(prim.copy(), t0=float(d[f"o{k}_time"][0]))   # undo the overlapped steps
        text = w.vtk_text(prim, float(d[f"o{k}_time"][0]), spec["variables"], grad)
        ref = files[f"sol{k:04d}_0.vtk"]
        assert len(text.splitlines()) == len(ref.splitlines())
        a, b = _numbers(text), _numbers(ref)
        assert a.shape == b.shape and np.allclose(a, b, rtol=1e-9, atol=1e-9 * np.max(np.abs(b)))


def test_output_needs_pinned_buffers():
    spec, cfg, mesh, prim0, d, files = _load("out_sq_euler")
    s = gpu.Solver(abi.Problem(preproc.preprocess(mesh), cfg))
    s.set_state(prim0)
    with pytest.raises(gpu.TensumError) as e:
        s.output_begin(np.empty((mesh.n_vertex, 5)))
    assert abi.STATUS[e.value.status] == "TG_INVALID_ARG"


@pytest.mark.parametrize("flux", ["kep", "kepec", "roe_ec"])
def test_central_flux_gradients_after_steps(flux):
    """Inviscid central-flux steps keep only V5 of the entropy variables; gradients
    asked for after steps (tg_gradients, an output snapshot) come from variables
    formed again from the state, bit for bit those of a handle given that state."""
    from tensum_b200 import cases
    g = preproc.preprocess(cases.kh_mesh(33, 0))
    a, phi = cases.kh_coefficients(1)
    P = abi.Problem(g, dict(flux=flux, reconstruct="first", boundary={t: ("periodic", {}) for t in (1, 2, 3, 4)},
                            final_time=1e9, time_stamps=1))
    s = gpu.Solver(P)
    s.set_state(cases.kh_ic(g.coords, a, phi))
    s.step(4)
    state = s.get_state()
    ref = gpu.Solver(P)
    ref.set_state(state)
    want = ref.gradients()
    prim, grad = s.output_buffers()
    s.output_begin(prim, grad, s.GRAD_CURRENT)
    s.output_wait()
    assert np.array_equal(prim, state) and np.array_equal(grad, want)
    assert np.array_equal(s.gradients(), want)
