"""Monte Carlo over the cylinder's uncertain inflow: batched FP32 and FP64 per sample.

The uncertain inputs of a sample are the free-stream Mach number, the
Reynolds number and the inflow angle; each sample runs the Navier-Stokes
cylinder (adiabatic no-slip wall, characteristic far field at its free
stream) from its uniform free stream to `final_time`, and the force on the
wall (compute_forces, src/force.cc:116-219) is recorded at `n_out` equally
spaced output times.  Its QoIs over the window t >= t_start are

    0: mean drag coefficient
    1: RMS of the lift-coefficient fluctuation
    2: mean viscous share of the drag

(`qoi.cylinder_qoi` adds the Strouhal number when shedding cycles fit the window).

`run_batched` advances all samples together in one FP32 batch (per-sample
viscosity and far-field values); `run_fp64` runs them through the FP64
single-solve handle, several handles on their own streams at once, which is
the fastest way this GPU runs independent FP64 samples.
"""
from __future__ import annotations

import threading
import time

import numpy as np

from . import abi, batch, cases, gpu, qoi

FORCES = {"cylinder": [1]}
NAMES = ("mean drag coefficient", "lift coefficient RMS", "viscous share of drag")


def draw_inputs(n: int, seed: int) -> np.ndarray:
    """(n, 3): Mach ~ U[0.15, 0.25], Re ~ U[80, 120], inflow angle ~ U[-2, 2] degrees."""
    r = np.random.default_rng(seed)
    return np.stack([r.uniform(0.15, 0.25, n), r.uniform(80.0, 120.0, n), r.uniform(-2.0, 2.0, n)], axis=1)


def qois(times, force_rows, mach: float, angle_deg: float, t_start: float) -> np.ndarray:
    """The three QoIs of one sample from its force history (rows inviscid x, y, viscous x, y)."""
    f = np.asarray(force_rows, np.float64)
    cd, cl = qoi.force_coefficients(f, mach, angle_deg)
    cdv, _ = qoi.force_coefficients(np.concatenate([np.zeros_like(f[:, :2]), f[:, 2:]], axis=1), mach, angle_deg)
    sel = np.asarray(times) >= t_start
    q = qoi.cylinder_qoi(times, cd, cl, mach, t_start)
    return np.array([q[0], q[1], float(np.mean(cdv[sel]) / np.mean(cd[sel]))])


def _configs(inputs, final_time, n_out, flux, recon):
    return [cases.cylinder_config(m, re, a, final_time, n_out, flux=flux, recon=recon) for m, re, a in inputs]


def run_batched(g, coords, inputs, final_time: float, n_out: int, t_start: float,
                flux: str = "kepes_tecno_roe", recon: str = "minmod", tune: bool = True, time_steps: int = 0) -> dict:
    """Every sample of `inputs` in one FP32 batch; returns QoIs (S, 3), the
    force histories, the wall time of the stepping and the steps issued, and
    (time_steps > 0) the device time per step of that many further steps."""
    S = inputs.shape[0]
    cfgs = _configs(inputs, final_time, n_out, flux, recon)
    b = batch.Batch([(abi.Problem(g, cfgs[0]), S)])
    b.set_parameters(0, mu_ref=[c["mu_ref"] for c in cfgs],
                     bface_values=np.stack([abi.bface_values(g, c["boundary"]) for c in cfgs]))
    ic = np.stack([cases.cylinder_ic(coords[:1], m, a)[0] for m, _, a in inputs])
    shape = None
    if tune:
        b.set_uniform(0, ic)
        shape, _ = b.tune(3)
    b.set_uniform(0, ic)
    hist = [b.forces(0, FORCES)[:, 0]]
    steps = 0
    t0 = time.perf_counter()
    for i in range(1, n_out + 1):
        info = b.advance(i)
        steps += int(info[0])
        hist.append(b.forces(0, FORCES)[:, 0])
    wall = time.perf_counter() - t0
    _, _, bad = b.clock(0)
    ms_step = None
    if time_steps > 0:
        b.set_uniform(0, ic)
        ms_step = b.time_steps(time_steps)
    hist = np.stack(hist, axis=1)                      # (S, n_out + 1, 4)
    times = np.linspace(0.0, final_time, n_out + 1)
    y = np.stack([qois(times, hist[s], inputs[s, 0], inputs[s, 2], t_start) for s in range(S)])
    return dict(y=y, forces=hist, times=times, wall_s=wall, steps=steps, bad=int(bad.sum()), shape=shape,
                kernels_per_step=int(b.query("kernels_per_step")), ms_per_step=ms_step)


def run_fp64(g, coords, inputs, final_time: float, n_out: int, t_start: float,
             flux: str = "kepes_tecno_roe", recon: str = "minmod", streams: int = 8) -> dict:
    """Every sample through the FP64 handle, `streams` handles stepping at
    once (one host thread each; the ABI calls release the interpreter).
    Returns QoIs (N, 3), force histories, wall time and steps per sample."""
    N = inputs.shape[0]
    cfgs = _configs(inputs, final_time, n_out, flux, recon)
    times = np.linspace(0.0, final_time, n_out + 1)
    hist = np.zeros((N, n_out + 1, 4))
    steps = np.zeros(N)
    solvers = [gpu.Solver(abi.Problem(g, cfgs[0])) for _ in range(min(streams, N))]
    errors = []

    def work(k):
        s64 = solvers[k]
        try:
            for s in range(k, N, len(solvers)):
                s64.update_parameters(abi.Problem(g, cfgs[s]))
                s64.set_state(cases.cylinder_ic(coords, inputs[s, 0], inputs[s, 2]))
                hist[s, 0] = s64.forces(FORCES)[0]
                for i in range(1, n_out + 1):
                    info = s64.advance(i)
                    hist[s, i] = s64.forces(FORCES)[0]
                steps[s] = info[3]
        except Exception as e:     # re-raised on the calling thread
            errors.append(e)

    th = [threading.Thread(target=work, args=(k,)) for k in range(len(solvers))]
    t0 = time.perf_counter()
    for t in th:
        t.start()
    for t in th:
        t.join()
    wall = time.perf_counter() - t0
    if errors:
        raise errors[0]
    y = np.stack([qois(times, hist[s], inputs[s, 0], inputs[s, 2], t_start) for s in range(N)])
    return dict(y=y, forces=hist, times=times, wall_s=wall, steps=steps, streams=len(solvers))
