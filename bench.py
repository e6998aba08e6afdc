"""Benchmark: vertex-stage updates/s of the FP64 explicit residual/update path.

Workload (one GPU) -- the Kelvin-Helmholtz configuration: a seeded, jittered
1025 x 1025 periodic triangulation of [0,1]^2 (1,050,625 stored vertices,
3,147,776 edges), density 2 / 1 shear layer with the seeded 10-mode velocity
perturbation, FP64, SSP-RK3, CFL 0.8, run with each of the four fluxes the
configuration names: KEP, KEPEC, Roe-EC and KEPES-TeCNO-Rusanov (minmod
reconstruction).  A "step" advances each of the four solves by one SSP-RK3
time step (3 stages); the value is the total vertex-stage updates of the four
solves divided by their total device time.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun each rank runs an independent replica (one partition per GPU;
the single solve does not shard), so scaling is weak and the value is the sum
over ranks divided by the slowest rank's time.

Keys beyond the base contract:
  per_flux      value, ms/step and roofline of each flux
  roofline      the dominant phase (the TeCNO-Rusanov flux pass) vs the measured HBM peak
  step_roofline whole time steps, per-flux algorithmic bytes
  cpu_baseline  the reference's own CPU code on this host (rank 0, N = 1)
  e2e           same metric through the C ABI with host buffers every step
  clocks        SM clock and throttle reasons sampled during the timed region

    python bench.py --workload mc [--samples S] [--n 257] [--steps K]

    python bench.py --workload cylinder [--samples S] [--final-time T] [--outputs K] [--t-start T0]

measures the surrogate control-variate configuration on the Navier-Stokes
cylinder (128 x 256 O-mesh; Mach ~ U[0.15, 0.25], Re ~ U[80, 120], angle ~
U[-2, 2] degrees): S batched FP32 solves to time T with the wall force at K
output times, FP64 solves of a subset (several handles at once), a surrogate
trained on the first --train solves, and the time to a 1 % relative standard
error of the mean and of the variance of each QoI for plain FP64 MC, batched
FP32 MC and batched FP32 with the control variate.  With --throughput-only
either Monte Carlo workload times the ensemble's graph-replayed steps alone
(a short command for a profiler).

    python bench.py --workload partitioned [--parts 1,2,4] [--steps K]

times the domain-decomposed single solve (tensum_b200.partition) on the same
Kelvin-Helmholtz workload: every partition on this one GPU, halos exchanged by
device copies, the whole step of all partitions replayed as one CUDA graph,
against the one-partition step, per flux and partition count.

--workload mc measures the Monte Carlo configuration instead: S Kelvin-Helmholtz samples
(rnd rows, device-generated initial states) on an n x n mesh advanced together
by the batched FP32 engine (KEPES-TeCNO-Rusanov, minmod), against the FP64
per-sample path on the same GPU, with the QoI error of the FP32 members
against FP64 runs and the time to a 1 % relative standard error of the mean
QoI for plain FP64 MC, batched FP32 MC and batched FP32 with the surrogate
control variate.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "vertex-stage updates/s"
UNIT = "vertex-stage updates/s"
FALLBACK_HBM_GBS = 6650.0
FLUXES = [("kep", "first"), ("kepec", "first"), ("roe_ec", "first"), ("kepes_tecno_rusanov", "minmod")]
DOMINANT = "kepes_tecno_rusanov"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=1025, help="vertices per side of the periodic mesh")
    ap.add_argument("--fluxes", default=",".join(f for f, _ in FLUXES),
                    help="comma-separated subset of kep,kepec,roe_ec,kepes_tecno_rusanov")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--e2e-steps", type=int, default=20)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="single",
                    choices=["single", "mc", "cylinder", "cylinder-rse", "cylinder2", "multilevel", "partitioned"])
    ap.add_argument("--samples", type=int, default=None,
                    help="ensemble size (--workload mc: 4096, --workload cylinder: 1024)")
    ap.add_argument("--final-time", type=float, default=2.0, help="cylinder: run length of every sample")
    ap.add_argument("--outputs", type=int, default=40, help="cylinder: force outputs over the run")
    ap.add_argument("--t-start", type=float, default=1.0, help="cylinder: start of the QoI window")
    ap.add_argument("--fp64-samples", type=int, default=32, help="cylinder: samples also run in FP64")
    ap.add_argument("--train", type=int, default=256, help="cylinder: solver runs the surrogate is trained on")
    ap.add_argument("--no-mc", action="store_true", help="skip the Monte Carlo object of the default line")
    ap.add_argument("--parts", default="1,2,4", help="partitioned: partition counts")
    ap.add_argument("--throughput-only", action="store_true", help="mc, cylinder: the ensemble's stepping alone")
    ap.add_argument("--mc-cap", type=float, default=120.0,
                    help="mc: wall-clock cap of the plain FP64 arm of the measured time to 1%% RSE "
                         "(cylinder-rse: of the plain and the batched arms)")
    ap.add_argument("--cv-cap", type=float, default=900.0,
                    help="cylinder-rse: wall-clock cap of the control-variate arm")
    a = ap.parse_args()
    a.flux_list = [(f, r) for f, r in FLUXES if f in a.fluxes.split(",")]
    return a


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def workload(args):
    from tensum_b200 import cases
    m = cases.kh_mesh(args.n, seed=args.seed)
    a, phi = cases.kh_coefficients(args.seed)
    prim0 = cases.kh_ic(m.coords, a, phi)
    return m, prim0


def flux_cfg(flux, recon):
    return dict(flux=flux, reconstruct=recon, boundary={t: ("periodic", {}) for t in (1, 2, 3, 4)},
                final_time=1.0e9, time_stamps=1, cfl=0.8)


def algorithmic_bytes(flux, V, E):
    """Compulsory HBM bytes per stage of the three-pass model (FP64, 2D, int32 indices).

    gradient pass: read U 32V, edges 24E, area 8V; write grad 64V
    flux pass:     read U 32V, grad 64V, coords 16V, edges 24E; write R 32V
    update pass:   read U, U_old, R 32V each, area 8V; write U 32V
    per step:      dt pass (U 32V, edges 24E, area 8V) + U_old write 32V, over 3 stages
    The central fluxes (KEP, KEPEC, Roe-EC) read no gradient, so for them the
    gradient pass and the gradient/coordinate reads of the flux pass drop out.
    """
    grad_pass = 104 * V + 24 * E
    flux_pass = 144 * V + 24 * E
    upd_pass = 136 * V
    dt_amort = (72 * V + 24 * E) / 3.0
    if flux.startswith("kepes_tecno"):
        stage = grad_pass + flux_pass + upd_pass + dt_amort
        fpass = flux_pass
    else:
        fpass = flux_pass - 80 * V
        stage = fpass + upd_pass + dt_amort
    return stage, fpass


def config_dict(args, m, n_edges):
    names = "+".join(f"{f}({r})" if r != "first" else f for f, r in args.flux_list)
    return {"workload": f"kelvin-helmholtz periodic {args.n}x{args.n}, each of {names}, ssprk3 cfl 0.8, fp64",
            "mesh_vertices": int(m.n_vertex), "mesh_edges": int(n_edges), "stages_per_step": 3,
            "solves_per_step": len(args.flux_list),
            "parallelism": "replicas" if args.gpus > 1 else "single", "l2": "working set > L2 (no flush needed)"}


# ----------------------------------------------------------------------------- clocks
class ClockSampler:
    """Polls NVML (SM clock, throttle reasons) on a thread while the timed region runs."""

    REASONS = {0x2: "applications_clocks_setting", 0x4: "sw_power_cap", 0x8: "hw_slowdown",
               0x10: "sync_boost", 0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown",
               0x80: "hw_power_brake_slowdown", 0x100: "display_clock_setting"}

    def __init__(self, device_index):
        self.samples = []
        self.reasons = 0
        self.max_mhz = None
        self._stop = threading.Event()
        self.ok = False
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(device_index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
            self.ok = True
        except Exception:
            self.ok = False

    def _run(self):
        while not self._stop.is_set():
            try:
                self.samples.append(self.nv.nvmlDeviceGetClockInfo(self.h, self.nv.NVML_CLOCK_SM))
                try:
                    r = self.nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                except Exception:
                    r = self.nv.nvmlDeviceGetCurrentClocksThrottleReasons(self.h)
                self.reasons |= int(r)
            except Exception:
                pass
            time.sleep(0.005)

    def __enter__(self):
        if self.ok:
            self.t = threading.Thread(target=self._run, daemon=True)
            self.t.start()
        return self

    def __exit__(self, *a):
        if self.ok:
            self._stop.set()
            self.t.join()

    def summary(self):
        if not self.ok or not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": [], "samples": 0}
        names = [n for b, n in self.REASONS.items() if self.reasons & b]
        return {"sm_mhz": float(statistics.median(self.samples)), "sm_max_mhz": self.max_mhz,
                "reasons": names, "samples": len(self.samples)}


# ----------------------------------------------------------------------------- reference arm
def reference_rate(args, m, prim0, steps, warm):
    """Time the reference's own CPU code (oracle/_ref harness) on the same workload, per flux."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_runner
    if not ref_runner.harness_available():
        return None
    total_s, total_vs, per = 0.0, 0, {}
    with tempfile.TemporaryDirectory(prefix="tensum_ref_bench_") as wd:
        for flux, recon in args.flux_list:
            d = ref_runner.run_case(m, flux_cfg(flux, recon), prim0, warm + steps, 0, workdir=wd, timeout=3600)
            st = d["step_s"][warm:]
            total_s += float(np.sum(st))
            total_vs += m.n_vertex * 3 * len(st)
            per[flux] = m.n_vertex * 3 * len(st) / float(np.sum(st))
    return {"value": total_vs / total_s, "unit": UNIT, "cores": 1, "kind": "reference", "seconds": total_s,
            "per_flux": per,
            "sample": f"{steps} SSP-RK3 step(s) of each flux on the full {args.n}x{args.n} workload after {warm} "
                      f"warm-up step(s); reference sources built -O3 with a serial MPI stub (one process, one core)"}


def run_reference(args):
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    m, prim0 = workload(args)
    steps = max(1, min(args.steps, 2))
    warm = 1 if args.warmup > 0 else 0
    r = reference_rate(args, m, prim0, steps, warm)
    from tensum_b200 import preproc
    ne = preproc.preprocess(m).n_face
    if r is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/tensum_harness is not built on this host"}))
        return 0
    line = {"metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": args.gpus, "steps": steps,
            "warmup": warm, "ms_per_step": 1e3 * r["seconds"] / steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded mesh and field)",
            "config": config_dict(args, m, ne), "impl": "reference", "per_flux": r["per_flux"],
            "steps_note": f"{steps} timed step(s) per flux (about {r['seconds'] / max(1, len(args.flux_list)) / steps:.1f} "
                          "s each on one core), fewer than the GPU arm's, which times --steps; the metric is a "
                          "rate, so the counts need not match",
            "cpu_baseline": {k: r[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": r["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ----------------------------------------------------------------------------- our arm
def traffic_from_profile(tag):
    """Per-launch DRAM bytes of the dominant phase from the committed ncu summary, if any."""
    try:
        for line in open(os.path.join(ROOT, "profiles", f"{tag}.txt")):
            if line.startswith("traffic_bytes_per_launch:"):
                return float(line.split(":", 1)[1])
    except OSError:
        pass
    return None


def run_ours(args):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    else:
        torch.cuda.set_device(0)
    dev = torch.cuda.current_device()

    from tensum_b200 import abi, gpu, preproc
    m, prim0 = workload(args)
    g = preproc.preprocess(m)
    V, E = g.n_vertex, g.n_face
    solvers = []
    for flux, recon in args.flux_list:
        s = gpu.Solver(abi.Problem(g, flux_cfg(flux, recon)))
        s.set_state(prim0)
        s.step(max(3, args.warmup))
        solvers.append((flux, s, torch.cuda.ExternalStream(s.stream_ptr())))
    torch.cuda.synchronize()
    if dist:
        dist.barrier()

    per, total_ms, launches = {}, 0.0, 0
    with ClockSampler(dev) as clk:
        for flux, s, stream in solvers:
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            ev0.record(stream)
            s.step(args.steps)
            ev1.record(stream)
            torch.cuda.synchronize()
            ms = ev0.elapsed_time(ev1)
            per[flux] = {"ms": ms}
            total_ms += ms
            launches += int(s.query("kernels_per_step")) * args.steps
    if dist:
        t = torch.tensor([total_ms] + [per[f]["ms"] for f, _, _ in solvers], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t[0])
        for i, (f, _, _) in enumerate(solvers):
            per[f]["ms"] = float(t[i + 1])
    nsolve = len(solvers)
    value = V * 3 * args.steps * nsolve * world / (total_ms / 1e3)
    peak, peak_kind = measured_peaks()
    for flux, s, _ in solvers:
        stage_b, fpass_b = algorithmic_bytes(flux, V, E)
        ms_step = per[flux]["ms"] / args.steps
        per[flux].update({"value": V * 3 * args.steps * world / (per[flux]["ms"] / 1e3), "ms_per_step": ms_step,
                          "step_roofline_frac": 3 * stage_b / (ms_step / 1e3) / 1e9 / peak,
                          "flux_pass_ms": s.time_phase("flux", 30)})
        per[flux]["flux_pass_frac"] = fpass_b / (per[flux]["flux_pass_ms"] / 1e3) / 1e9 / peak
        if flux.startswith("kepes_tecno"):
            per[flux]["gradient_ms"] = s.time_phase("gradient", 30)
        del per[flux]["ms"]
    dom = per.get(DOMINANT) or next(iter(per.values()))
    dom_flux = DOMINANT if DOMINANT in per else next(iter(per))
    _, fpass_b = algorithmic_bytes(dom_flux, V, E)
    roof = {"bound": "hbm", "kernel": f"{dom_flux} flux pass (tiled edge fluxes + residual gather)",
            "achieved": fpass_b / (dom["flux_pass_ms"] / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
            "frac": fpass_b / (dom["flux_pass_ms"] / 1e3) / 1e9 / peak,
            "traffic": traffic_from_profile("flux_pass_kh1025"), "algorithmic_bytes_per_launch": fpass_b,
            "ms_per_launch": dom["flux_pass_ms"], "peak_source": peak_kind}
    step_bytes = sum(3 * algorithmic_bytes(f, V, E)[0] for f, _, _ in solvers)
    step_roof = {"achieved": step_bytes * args.steps / (total_ms / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                 "frac": step_bytes * args.steps / (total_ms / 1e3) / 1e9 / peak,
                 "bytes_per_step": step_bytes, "model": "408V+56E per stage (TeCNO), 224V+32E (central fluxes)"}

    # end to end through the C ABI with host buffers every step (dominant flux):
    # PrimVar records in and out of pinned host memory, pipelined (the next
    # step's state streams in by tg_set_state_async and the last result streams
    # out by tg_output_begin while the device steps); for comparison the
    # blocking calls, from pinned (DMA) and from pageable numpy arrays (the
    # library's staging ring)
    s_e2e = dict((f, s) for f, s, _ in solvers)[dom_flux]
    pin_in = torch.empty((V, 5), dtype=torch.float64, pin_memory=True).numpy()
    pin_out = torch.empty((V, 5), dtype=torch.float64, pin_memory=True).numpy()
    pin_in2 = torch.empty((V, 5), dtype=torch.float64, pin_memory=True).numpy()
    pin_out2 = torch.empty((V, 5), dtype=torch.float64, pin_memory=True).numpy()
    pin_in[:] = prim0
    pin_in2[:] = prim0
    page_out = np.empty((V, 5))
    ne2e = max(1, min(args.e2e_steps, args.steps))

    def e2e_run(src, dst):
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(ne2e):
            s_e2e.set_state(src)
            s_e2e.step(1)
            s_e2e.get_state(out=dst)
        el = time.perf_counter() - t0
        if dist:
            t = torch.tensor([el], device="cuda", dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            el = float(t.item())
        return V * 3 * ne2e * world / el

    def e2e_pipelined(s):
        """Seconds for ne2e steps of solver s with its state in and out of host memory each step."""
        ins, outs = (pin_in, pin_in2), (pin_out, pin_out2)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        s.set_state_async(ins[0])
        for i in range(ne2e):
            if i + 1 < ne2e:
                s.set_state_async(ins[(i + 1) % 2])   # the next step's input streams in now
            s.step(1)                                 # takes this step's input, steps
            s.output_begin(outs[i % 2])               # the result streams out during the next step
        s.output_wait()
        el = time.perf_counter() - t0
        if dist:
            t = torch.tensor([el], device="cuda", dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            el = float(t.item())
        return el

    # the same four solves as `value`: every flux ne2e steps, total updates over total time
    e2e_run(pin_in, pin_out)   # first touch of the staging paths
    e2e_pipelined(s_e2e)
    e2e_s = {f: e2e_pipelined(s) for f, s, _ in solvers}
    e2e = {"value": V * 3 * ne2e * world * len(e2e_s) / sum(e2e_s.values()), "unit": UNIT,
           "h2d_bytes_per_step": 40 * V * len(e2e_s), "d2h_bytes_per_step": 40 * V * len(e2e_s), "steps": ne2e,
           "fluxes": list(e2e_s), "per_flux": {f: V * 3 * ne2e * world / t for f, t in e2e_s.items()},
           "path": "per step and flux: tg_set_state_async(pinned host PrimVar[V]) of the next step's input, "
                   "tg_step(1), tg_output_begin(pinned host PrimVar[V]) of its result; copies overlap the steps",
           "blocking_flux": dom_flux,
           "blocking_value": e2e_run(pin_in, pin_out),
           "blocking_path": "tg_set_state(pinned) + tg_step(1) + tg_get_state(pinned) per step",
           "pageable_value": e2e_run(np.ascontiguousarray(prim0), page_out)}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        r = reference_rate(args, m, prim0, 1, 1)
        if r is not None:
            cpu = {k: r[k] for k in ("value", "unit", "cores", "kind", "sample", "per_flux")}

    mc = None
    if rank == 0 and world == 1 and not args.no_mc:
        solvers.clear()          # release the single-solve handles before the ensemble
        s_e2e = None
        mc = mc_line(257, 4096, 20, 3, args.seed, mc_cap=args.mc_cap)
        mc = {k: mc[k] for k in ("metric", "value", "unit", "ms_per_step", "config", "autotune", "fp64_per_sample",
                                 "roofline", "qoi", "time_to_rse_measured", "time_to_rse", "cv", "clocks")}
        mc["command"] = "python bench.py --workload mc --steps 20 --warmup 3"

    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": max(3, args.warmup), "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded mesh and field)",
            "config": config_dict(args, m, E), "per_flux": per, "roofline": roof, "step_roofline": step_roof,
            "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches, "clocks": clk.summary(), "impl": "ours",
            "mc": mc}
    print(json.dumps(line))
    return 0


# ----------------------------------------------------------------------------- Monte Carlo workload
MC_BYTES_PER_VSS = 187.0   # FP32 batched compulsory bytes per vertex-sample-stage (state, U_old, gradients)


def mc_line(n, S, K, W, seed, throughput_only=False, mc_cap=120.0):
    """Batched FP32 ensemble throughput and time to QoI error (one GPU): the JSON object
    (throughput_only: the graph-replayed steps alone, e.g. for a profiler)."""
    import torch
    from tensum_b200 import abi, batch, cases, cv, gpu, mlp, preproc
    torch.cuda.set_device(0)
    m = cases.kh_mesh(n, seed)
    V = m.n_vertex
    g = preproc.preprocess(m)
    base = dict(flux="kepes_tecno_rusanov", reconstruct="minmod", boundary={t: ("periodic", {}) for t in (1, 2, 3, 4)},
                cfl=0.8, time_stamps=1)
    t_q = 0.05                                     # QoI time for the accuracy and time-to-error parts
    rows = np.stack([cases.kh_rnd_row(seed * 1000003 + s) for s in range(S)])

    # throughput: K graph-replayed steps of every sample (final time far away)
    P_long = abi.Problem(g, dict(base, final_time=1.0e9))
    b = batch.Batch([(P_long, S)])
    b.set_kh(0, rows)
    shape, tune_ms = b.tune(3)
    b.time_steps(W)
    with ClockSampler(0) as clk:
        ms = b.time_steps(K) * K           # CUDA events on the batch's stream around K graph replays
    value = V * S * 3 * K / (ms / 1e3)
    launches = int(b.query("kernels_per_step")) * K
    del b
    peak, peak_kind = measured_peaks()
    if throughput_only:
        return {"metric": "vertex-sample-stage updates/s (FP32 ensemble)", "value": value,
                "unit": "vertex-sample-stage updates/s", "ms_per_step": ms / K, "steps": K, "gpu_launches": launches,
                "config": {"workload": f"kelvin-helmholtz {n}x{n} periodic ensemble of {S} samples, "
                                       "kepes_tecno_rusanov(minmod), ssprk3, fp32 members", "shape": shape},
                "clocks": clk.summary()}

    # FP64 per-sample path on the same mesh
    s64 = gpu.Solver(P_long)
    s64.set_state(cases.kh_ic_rnd(m.coords, rows[0]))
    s64.step(W)
    ms64 = s64.time_phase("step", max(20, K))
    del s64

    # QoIs at t_q: every sample batched, a subset in FP64
    P_q = abi.Problem(g, dict(base, final_time=t_q))
    bq = batch.Batch([(P_q, S)])
    bq.set_kh(0, rows)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    info = bq.advance(1)
    torch.cuda.synchronize()
    t_batch = time.perf_counter() - t0
    y = bq.integrals(0)
    n_sub = 32
    s64 = gpu.Solver(P_q)
    y64, steps64 = [], []
    w = np.ones(V)
    for st in m.periodic_sets:
        w[st] = 1.0 / len(st)
    aw = g.dcarea * w
    t0 = time.perf_counter()
    for s in range(n_sub):
        s64.set_state(cases.kh_ic_rnd(m.coords, rows[s]))
        inf = s64.advance(1)
        steps64.append(inf[3])
        q = s64.get_state()
        rho = q[:, 1] / q[:, 0]
        ent = np.log(q[:, 1]) - 1.4 * np.log(rho)
        y64.append([np.sum(0.5 * rho * q[:, 3] ** 2 * aw), np.sum(0.5 * rho * q[:, 2] ** 2 * aw),
                    np.sum(-rho * ent / 0.4 * aw)])
    t_fp64_sample = (time.perf_counter() - t0) / n_sub
    y64 = np.array(y64)
    qerr = np.abs(y[:n_sub] - y64) / np.abs(y64)
    fm32, _, m232 = bq.moments(0)
    del bq

    # time to a 1 % relative standard error of the mean of q0 (vertical kinetic energy)
    n_train = min(1024, S // 4)
    net = mlp.MLP(rows.shape[1], 3, seed=1)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    net.fit(rows[:n_train], y[:n_train], epochs=300, batch=128, lr=2e-3)
    t_train = time.perf_counter() - t0
    x_extra = np.random.default_rng(10 ** 7 + seed).uniform(0.0, 1.0, size=(1 << 20, rows.shape[1]))
    t0 = time.perf_counter()
    g_extra = net.predict(x_extra, precision=1)
    t_surr = time.perf_counter() - t0
    g_ev = net.predict(rows[n_train:], precision=1)
    r = cv.estimate(y[n_train:], g_ev, g_extra)
    t_batch_sample = t_batch / S
    ttr = {}
    for rse in (0.01, 0.001):
        n_plain = float(cv.samples_for_rse(y[n_train:, 0], None, rse)[0])
        n_cv = float(cv.samples_for_rse(y[n_train:, 0], g_ev[:, 0], rse)[0])
        t = {"plain_fp64_mc_s": n_plain * t_fp64_sample, "batched_fp32_mc_s": n_plain * t_batch_sample,
             "batched_fp32_cv_s": (n_train + n_cv) * t_batch_sample + t_train + t_surr}
        ttr[f"rse_{rse:g}"] = dict(t, samples_plain=n_plain, samples_cv=n_cv,
                                   speedup_batched_vs_plain_fp64=t["plain_fp64_mc_s"] / t["batched_fp32_mc_s"],
                                   speedup_cv_vs_plain_fp64=t["plain_fp64_mc_s"] / t["batched_fp32_cv_s"])
    # measured: each arm sampled until the mean and variance of every QoI reach 1 % RSE
    from tensum_b200 import mcrse
    measured = mcrse.measure(g, m, dict(base, final_time=t_q), lambda i: cases.kh_rnd_row(seed * 1000003 + i),
                             rse=0.01, cap_s=mc_cap, seed=seed)
    line = {"metric": "vertex-sample-stage updates/s (FP32 ensemble); time to 1% RSE of the mean QoI vs plain FP64 MC",
            "value": value, "unit": "vertex-sample-stage updates/s", "n_gpus": 1, "steps": K, "warmup": W,
            "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 members, f64 geometry / log-mean series / moments", "data": "synthetic (seeded rnd rows)",
            "config": {"workload": f"kelvin-helmholtz {n}x{n} periodic ensemble of {S} samples, kepes_tecno_rusanov(minmod), "
                                   "ssprk3 cfl 0.8", "mesh_vertices": V, "samples": S,
                       "l2": "working set > L2 (no flush needed)"},
            "autotune": {"shape": shape, "ms_per_step_by_shape": [float(x) for x in tune_ms]},
            "fp64_per_sample": {"ms_per_step": ms64, "value": V * 3 / (ms64 / 1e3),
                                "batched_speedup_per_sample_stage": value / (V * 3 / (ms64 / 1e3))},
            "roofline": {"bound": "hbm", "kernel": "whole batched step", "bytes_per_vertex_sample_stage": MC_BYTES_PER_VSS,
                         "achieved": MC_BYTES_PER_VSS * value / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": MC_BYTES_PER_VSS * value / 1e9 / peak, "traffic": None, "peak_source": peak_kind},
            "qoi": {"time": t_q, "names": ["0.5 rho v^2", "0.5 rho u^2", "-rho s/(gamma-1)"],
                    "fp32_vs_fp64_rel_err_max": [float(x) for x in qerr.max(0)], "fp64_subset": n_sub,
                    "batched_steps_issued": float(info[0]), "fp64_steps_mean": float(np.mean(steps64))},
            "time_to_rse_measured": dict(measured, qoi_time=t_q,
                                         qois=["0.5 rho v^2", "0.5 rho u^2", "-rho s/(gamma-1)"]),
            "time_to_rse": dict(ttr, qoi="0.5 rho v^2 (mean)", n_train=n_train, train_s=t_train,
                                surrogate_evals=1 << 20, surrogate_eval_s=t_surr,
                                fp64_sample_s=t_fp64_sample, batched_sample_s=t_batch_sample,
                                note="model: sample counts from the ensemble's variance and control-variate "
                                     "residual variance times per-sample costs (FP64 on a 32-sample subset); "
                                     "time_to_rse_measured holds the measured runs"),
            "cv": {"gain": [float(x) for x in r["gain"]], "used": [bool(x) for x in r["used"]],
                   "mean": [float(x) for x in r["mean"]], "plain_mean": [float(x) for x in r["plain_mean"]],
                   "se_mean": [float(x) for x in r["se_mean"]]},
            "gpu_launches": launches, "clocks": clk.summary(), "impl": "ours",
            "e2e": {"value": V * S * 3 * float(info[0]) / t_batch, "unit": "vertex-sample-stage updates/s",
                    "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0,
                    "path": "tg_batch_advance to the QoI time, wall clock, inputs generated on the device from rnd rows"}}
    return line


def run_mc(args):
    n = args.n if args.n != 1025 else 257
    print(json.dumps(mc_line(n, args.samples or 4096, args.steps, max(3, args.warmup), args.seed, mc_cap=args.mc_cap,
                             throughput_only=args.throughput_only)))
    return 0


def cylinder_line(S, T, n_out, t_start, n_fp64, n_train, K, seed, n_r=128, n_t=256, throughput_only=False):
    """Surrogate control-variate MC on the Navier-Stokes cylinder (one GPU): the JSON object
    (throughput_only: the ensemble's graph-replayed steps alone, e.g. for a profiler)."""
    import torch
    from tensum_b200 import cases, cv, cylinder, mlp, preproc
    torch.cuda.set_device(0)
    m = cases.cylinder_mesh(n_r, n_t, seed)
    V = m.n_vertex
    g = preproc.preprocess(m)
    X = cylinder.draw_inputs(S, seed)
    if throughput_only:
        with ClockSampler(0) as clk:
            rb = cylinder.run_batched(g, m.coords, X, 0.01, 1, 0.0, time_steps=K)
        return {"metric": "vertex-sample-stage updates/s (FP32 ensemble)", "value": V * S * 3 / (rb["ms_per_step"] / 1e3),
                "unit": "vertex-sample-stage updates/s", "ms_per_step": rb["ms_per_step"], "steps": K,
                "gpu_launches": rb["kernels_per_step"] * K,
                "config": {"workload": f"navier-stokes cylinder {n_r}x{n_t} O-mesh ensemble of {S} samples, "
                                       "kepes_tecno_roe(minmod), ssprk3, fp32 members", "shape": rb["shape"]},
                "clocks": clk.summary()}
    with ClockSampler(0) as clk:
        rb = cylinder.run_batched(g, m.coords, X, T, n_out, t_start, time_steps=K)
    y = rb["y"]
    r64 = cylinder.run_fp64(g, m.coords, X[:n_fp64], T, n_out, t_start)
    y64 = r64["y"]
    steps_per_sample = float(np.mean(r64["steps"]))
    t_b = rb["wall_s"] / S
    t_64 = r64["wall_s"] / n_fp64
    err = np.abs(y[:n_fp64] - y64) / np.maximum(np.abs(y64), 1e-300)
    mean_err = np.abs(y[:n_fp64].mean(0) - y64.mean(0)) / np.abs(y64.mean(0))
    std_err = np.abs(y[:n_fp64].std(0, ddof=1) - y64.std(0, ddof=1)) / y64.std(0, ddof=1)

    net = mlp.MLP(3, 3, seed=1)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    net.fit(X[:n_train], y[:n_train], epochs=400, batch=64, lr=2e-3)
    t_train = time.perf_counter() - t0
    x_extra = cylinder.draw_inputs(1 << 20, 10 ** 7 + seed)
    t0 = time.perf_counter()
    g_extra = net.predict(x_extra, precision=1)
    t_surr = time.perf_counter() - t0
    g_ev = net.predict(X[n_train:], precision=1)
    est = cv.estimate(y[n_train:], g_ev, g_extra)
    ttr = {}
    for rse in (0.01,):
        n_plain_mean = cv.samples_for_rse(y[n_train:], None, rse)
        n_cv_mean = cv.samples_for_rse(y[n_train:], g_ev, rse)
        n_plain_var = cv.samples_for_rse_var(y[n_train:], None, rse)
        n_cv_var = cv.samples_for_rse_var(y[n_train:], g_ev, rse)
        n_plain = float(max(n_plain_mean.max(), n_plain_var.max()))
        n_cv = float(max(n_cv_mean.max(), n_cv_var.max()))
        t = {"plain_fp64_mc_s": n_plain * t_64, "batched_fp32_mc_s": n_plain * t_b,
             "batched_fp32_cv_s": (n_train + n_cv) * t_b + t_train + t_surr}
        ttr[f"rse_{rse:g}"] = dict(
            t, samples_plain=n_plain, samples_cv=n_cv,
            samples_by_qoi={"plain_mean": n_plain_mean.tolist(), "cv_mean": n_cv_mean.tolist(),
                            "plain_var": n_plain_var.tolist(), "cv_var": n_cv_var.tolist()},
            speedup_batched_vs_plain_fp64=t["plain_fp64_mc_s"] / t["batched_fp32_mc_s"],
            speedup_cv_vs_plain_fp64=t["plain_fp64_mc_s"] / t["batched_fp32_cv_s"])
    value = V * 3 * S * steps_per_sample / rb["wall_s"]
    line = {"metric": "time to 1% RSE of the QoI mean and variance vs plain FP64 MC (cylinder, surrogate control variate)",
            "value": value, "unit": "vertex-sample-stage updates/s", "n_gpus": 1, "steps": rb["steps"], "warmup": 0,
            "ms_per_step": rb["ms_per_step"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 members, f64 geometry / log-mean series / forces / moments",
            "data": "synthetic (seeded uncertain inputs, seeded O-mesh)",
            "config": {"workload": f"navier-stokes cylinder {n_r}x{n_t} O-mesh, {S} samples, kepes_tecno_roe(minmod), "
                                   f"ssprk3 cfl 0.8, t = 0 .. {T}, forces at {n_out} outputs, QoI window t >= {t_start}",
                       "mesh_vertices": V, "samples": S, "final_time": T, "outputs": n_out, "t_start": t_start,
                       "inputs": "mach U[0.15,0.25], re U[80,120], angle U[-2,2] deg",
                       "l2": "working set > L2 (no flush needed)"},
            "qoi": {"names": list(cylinder.NAMES), "fp64_subset": n_fp64,
                    "fp32_vs_fp64_rel_err_max": err.max(0).tolist(), "fp32_vs_fp64_rel_err_mean": err.mean(0).tolist(),
                    "subset_mean_rel_err": mean_err.tolist(), "subset_std_rel_err": std_err.tolist(),
                    "ensemble_mean": y.mean(0).tolist(), "ensemble_std": y.std(0, ddof=1).tolist(),
                    "strouhal": "no shedding cycle fits the window (shedding needs t of order 100)"},
            "time_to_rse": dict(ttr, n_train=n_train, train_s=t_train, surrogate_evals=1 << 20,
                                surrogate_eval_s=t_surr, fp64_sample_s=t_64, fp64_streams=r64["streams"],
                                batched_sample_s=t_b,
                                note="sample counts from the ensemble's variance and the control-variate residual "
                                     "variance (mean and variance targets of all three QoIs); FP64 per-sample time "
                                     "measured on the FP64 subset run as concurrent handles"),
            "cv": {"gain": [float(x) for x in est["gain"]], "used": [bool(x) for x in est["used"]],
                   "mean": est["mean"].tolist(), "plain_mean": est["plain_mean"].tolist(),
                   "var": est["var"].tolist(), "plain_var": est["plain_var"].tolist(),
                   "se_mean": est["se_mean"].tolist()},
            "batched": {"wall_s": rb["wall_s"], "steps_issued": rb["steps"], "bad_samples": rb["bad"],
                        "shape": rb["shape"], "device_value": V * 3 * S / (rb["ms_per_step"] / 1e3)},
            "fp64": {"wall_s": r64["wall_s"], "steps_per_sample": steps_per_sample},
            "gpu_launches": rb["kernels_per_step"] * rb["steps"], "clocks": clk.summary(), "impl": "ours",
            "roofline": None,
            "e2e": {"value": value, "unit": "vertex-sample-stage updates/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0,
                    "path": "tg_batch_advance + tg_batch_forces at every output time, wall clock"}}
    return line


def run_cylinder(args):
    print(json.dumps(cylinder_line(args.samples or 1024, args.final_time, args.outputs, args.t_start, args.fp64_samples,
                                   args.train, max(5, min(args.steps, 50)), args.seed,
                                   throughput_only=args.throughput_only)))
    return 0


def cylinder2_line(n_steps, n_out, fp32_samples, seed, n_r=256, n_t=512, mach=0.2, reynolds=100.0):
    """The Navier-Stokes cylinder of the single-solve configuration (256 x 512 O-mesh, Mach 0.2,
    Re 100, adiabatic wall, characteristic far field) for n_steps SSP-RK3 steps in FP64 and, as an
    FP32 batch of identical members, over the same output times: the JSON object."""
    import torch
    from tensum_b200 import abi, batch, cases, cylinder, gpu, preproc, qoi
    torch.cuda.set_device(0)
    m = cases.cylinder_mesh(n_r, n_t, seed)
    g = preproc.preprocess(m)
    V = g.n_vertex
    ic = cases.cylinder_ic(m.coords, mach, 0.0)
    # the run length: n_steps steps at the time step the flow settles to (measured over a
    # first stretch), cut into n_out equal output intervals that both precisions stop at
    probe = gpu.Solver(abi.Problem(g, cases.cylinder_config(mach, reynolds, 0.0, 1.0e9, 1)))
    probe.set_state(ic)
    probe.step(1000)
    t1 = probe.step(1000)[0]
    ms64 = probe.time_phase("step", 200)      # device time of a step (final time far away)
    probe.close()
    T = float(n_steps * (t1 / 2000.0))
    cfg = cases.cylinder_config(mach, reynolds, 0.0, T, n_out)
    s = gpu.Solver(abi.Problem(g, cfg))
    s.set_state(ic)
    hist64 = [s.forces(cylinder.FORCES)[0]]
    with ClockSampler(0) as clk64:
        t0 = time.perf_counter()
        for i in range(1, n_out + 1):
            info = s.advance(i)
            hist64.append(s.forces(cylinder.FORCES)[0])
        wall64 = time.perf_counter() - t0
    steps64 = int(info[3])
    s.close()
    hist64 = np.array(hist64)
    times = np.linspace(0.0, T, n_out + 1)
    t_start = 0.5 * T
    cd64, cl64 = qoi.force_coefficients(hist64, mach, 0.0)
    q64 = qoi.cylinder_qoi(times, cd64, cl64, mach, t_start)
    # FP32 members: fp32_samples copies of the same configuration in one batch
    b = batch.Batch([(abi.Problem(g, cfg), fp32_samples)])
    rec = cases.cylinder_ic(m.coords[:1], mach, 0.0)
    b.set_uniform(0, np.repeat(rec, fp32_samples, axis=0))
    hist32 = [b.forces(0, cylinder.FORCES)[:, 0]]
    with ClockSampler(0) as clk32:
        t0 = time.perf_counter()
        for i in range(1, n_out + 1):
            b.advance(i)
            hist32.append(b.forces(0, cylinder.FORCES)[:, 0])
        wall32 = time.perf_counter() - t0
    _, _, bad = b.clock(0)
    hist32 = np.stack(hist32, axis=1)[0]
    cd32, cl32 = qoi.force_coefficients(hist32, mach, 0.0)
    q32 = qoi.cylinder_qoi(times, cd32, cl32, mach, t_start)
    sel = times >= t_start
    fl = cl64[sel] - cl64[sel].mean()
    # periodic shedding behind a circular cylinder at Re 100 carries a lift amplitude of
    # order 0.3 (RMS about 0.2); lift crossings at a far smaller amplitude are not shedding
    shed = bool(np.isfinite(q64[2]) and q64[1] > 0.01)
    err = np.abs(q32 - q64) / np.maximum(np.abs(q64), 1e-300)
    line = {"metric": "vertex-stage updates/s (navier-stokes cylinder, fp64) and the cylinder QoIs",
            "value": V * 3 * steps64 / wall64, "unit": UNIT, "n_gpus": 1, "steps": steps64, "warmup": 0,
            "ms_per_step": ms64, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded O-mesh, uniform free stream start)",
            "config": {"workload": f"navier-stokes cylinder {n_r}x{n_t} O-mesh (r 0.5..20, first spacing 2e-3, "
                                   f"ratio 1.02), mach {mach}, re {reynolds}, pr 0.72, adiabatic no-slip wall, "
                                   f"characteristic far field, kepes_tecno_roe(minmod), ssprk3 cfl 0.8, "
                                   f"{n_steps} steps to t = {T:.4g}, forces at {n_out} outputs",
                       "mesh_vertices": V, "final_time": T, "outputs": n_out, "qoi_window": [t_start, T]},
            "qoi": {"names": ["mean drag coefficient", "lift coefficient RMS", "strouhal number"],
                    "fp64": [float(x) for x in q64], "fp32": [float(x) for x in q32],
                    "fp32_vs_fp64_rel_err": [float(x) for x in err],
                    "shedding": shed,
                    "lift_upward_zero_crossings_in_window": int(np.count_nonzero((fl[:-1] < 0) & (fl[1:] >= 0))),
                    "lift_history_last_quarter": [float(x) for x in cl64[-(n_out // 4):][::max(1, n_out // 200)]],
                    "note": ("shedding measured in the window" if shed else
                             f"measured: no vortex shedding by t = {T:.4g} from the uniform start (lift RMS "
                             f"{q64[1]:.2g} against about 0.2 for a shedding cylinder at Re 100); the Strouhal "
                             "entry is that of the small lift oscillation, not of shedding")},
            "fp64": {"wall_s": wall64, "steps": steps64, "device_ms_per_step": ms64,
                     "device_value": V * 3 / (ms64 / 1e3), "clocks": clk64.summary()},
            "fp32": {"wall_s": wall32, "samples": fp32_samples, "bad_samples": int(bad.sum()),
                     "value": V * 3 * fp32_samples * steps64 / wall32, "clocks": clk32.summary()},
            "gpu_launches": None, "impl": "ours", "roofline": None, "clocks": clk64.summary(),
            "command": f"python bench.py --workload cylinder2 --steps {n_steps} --outputs {n_out}"}
    return line


def run_cylinder2(args):
    print(json.dumps(cylinder2_line(args.steps if args.steps != 200 else 200000, args.outputs if args.outputs != 40
                                    else 2000, args.samples or 32, args.seed)))
    return 0


def multilevel_line(levels, n_steps, n_fp64, seed):
    """The multilevel Monte Carlo configuration: Kelvin-Helmholtz ensembles on several meshes
    ((n, samples) per level) in one fused FP32 batch, all to the time the finest mesh reaches in
    n_steps steps; the pointwise mean and standard-deviation fields of the first n_fp64 samples of
    every level against FP64 solves of the same samples.  The JSON object."""
    import torch
    from tensum_b200 import abi, batch, cases, gpu, preproc
    torch.cuda.set_device(0)
    base = dict(flux="kepes_tecno_rusanov", reconstruct="minmod", boundary={t: ("periodic", {}) for t in (1, 2, 3, 4)},
                cfl=0.8)
    meshes = [cases.kh_mesh(n, seed + i) for i, (n, _) in enumerate(levels)]
    geoms = [preproc.preprocess(m) for m in meshes]
    rows = [np.stack([cases.kh_rnd_row(seed * 1000003 + 7919 * i + s) for s in range(S)])
            for i, (_, S) in enumerate(levels)]
    # common final time: n_steps of the finest level's first time step
    fine = int(np.argmax([g.n_vertex for g in geoms]))
    probe = gpu.Solver(abi.Problem(geoms[fine], dict(base, final_time=1.0e9, time_stamps=1)))
    probe.set_state(cases.kh_ic_rnd(meshes[fine].coords, rows[fine][0]))
    T = float(n_steps * probe.step(1)[1])
    probe.close()
    probs = [abi.Problem(g, dict(base, final_time=T, time_stamps=1)) for g in geoms]
    b = batch.Batch([(P, S) for P, (_, S) in zip(probs, levels)])
    for i, r in enumerate(rows):
        b.set_kh(i, r)
    shape, _ = b.tune(3)
    for i, r in enumerate(rows):
        b.set_kh(i, r)
    ms_step = b.time_steps(10)        # device time of a step of every level (graph replays)
    for i, r in enumerate(rows):
        b.set_kh(i, r)
    with ClockSampler(0) as clk:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        info = b.advance(1)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
    launches_steps = int(info[0])
    per_level, work = [], 0
    for i, ((n, S), g, m, P) in enumerate(zip(levels, geoms, meshes, probs)):
        el, cnt, bad = b.clock(i)
        # FP64 solves of the first n_fp64 samples of the level, to the same time
        k = min(n_fp64, S)
        s64 = gpu.Solver(P)
        x64, x32, steps64 = [], [], []
        for j in range(k):
            s64.set_state(cases.kh_ic_rnd(m.coords, rows[i][j]))
            inf = s64.advance(1)
            steps64.append(int(inf[3]))
            x64.append(s64.get_state())
            x32.append(b.get_state(i, j))
        s64.close()
        x64, x32 = np.stack(x64), np.stack(x32)
        cols = [0, 1, 2, 3]                      # T, p, u, v
        m64, m32 = x64.mean(0)[:, cols], x32.mean(0)[:, cols]
        sd64, sd32 = x64.std(0, ddof=1)[:, cols], x32.std(0, ddof=1)[:, cols]
        scale = np.abs(m64).max(0)
        scale[2] = scale[3] = max(scale[2], scale[3])
        work += g.n_vertex * S * 3 * int(np.mean(steps64))
        per_level.append({"n": n, "vertices": g.n_vertex, "samples": S, "steps": int(np.mean(steps64)),
                          "bad_samples": int(bad.sum()), "reached": bool(np.all(cnt >= 2)),
                          "fp64_subset": k,
                          "mean_field_rel_err": (np.abs(m32 - m64).max(0) / scale).tolist(),
                          "std_field_rel_err": (np.abs(sd32 - sd64).max(0) / (sd64.max(0) + 1e-300)).tolist()})
    line = {"metric": "vertex-sample-stage updates/s (multilevel FP32 ensemble, one fused batch)",
            "value": work / wall, "unit": "vertex-sample-stage updates/s", "n_gpus": 1, "steps": launches_steps,
            "warmup": 0, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 members, f64 geometry / log-mean series / clocks", "data": "synthetic (seeded rnd rows)",
            "config": {"workload": "kelvin-helmholtz multilevel ensemble " +
                                   ", ".join(f"{S} x {n}^2" for n, S in levels) +
                                   f", one fused batch, kepes_tecno_rusanov(minmod), ssprk3 cfl 0.8, to t = {T:.4g} "
                                   f"({n_steps} steps of the finest mesh)", "shape": shape, "final_time": T},
            "levels": per_level,
            "fields": "pointwise mean and sample standard deviation of T, p, u, v over the FP64 subset, "
                      "FP32 members against FP64 solves of the same samples; errors relative to each field's "
                      "maximum (velocities: the larger velocity scale)",
            "wall_s": wall, "gpu_launches": int(b.query("kernels_per_step")) * launches_steps,
            "clocks": clk.summary(), "impl": "ours", "roofline": None,
            "command": "python bench.py --workload multilevel"}
    return line


def run_multilevel(args):
    levels = [(129, 2048), (257, 512), (513, 128)]
    if args.samples:
        levels = [(n, max(32, (S * args.samples // 4096) // 32 * 32)) for n, S in levels]
    print(json.dumps(multilevel_line(levels, args.steps if args.steps != 200 else 1000, args.fp64_samples, args.seed)))
    return 0


def cylinder_rse_line(T, n_out, t_start, seed, cap_plain, cap_batched, cap_cv, n_r=128, n_t=256):
    """Measured time to 1 % RSE of the mean and variance of the cylinder QoIs for plain FP64 MC,
    batched FP32 MC and batched FP32 with the surrogate control variate: the JSON object."""
    import torch
    from tensum_b200 import cases, mcrse, preproc
    torch.cuda.set_device(0)
    m = cases.cylinder_mesh(n_r, n_t, seed)
    g = preproc.preprocess(m)
    with ClockSampler(0) as clk:
        r = mcrse.measure_cylinder(g, m.coords, T, n_out, t_start, rse=0.01, seed=seed, cap_plain_s=cap_plain,
                                   cap_batched_s=cap_batched, cap_cv_s=cap_cv)
    return {"metric": "wall time to 1% RSE of the mean and variance of the cylinder QoIs, vs plain FP64 MC",
            "value": r["speedup_cv_vs_plain_fp64"], "unit": "x (plain FP64 MC time / batched FP32 + CV time)",
            "higher_is_better": True, "n_gpus": 1, "dtype": "f32 members, f64 geometry / forces; fp64 plain arm",
            "data": "synthetic (seeded uncertain inputs, seeded O-mesh)",
            "config": {"workload": f"navier-stokes cylinder {n_r}x{n_t} O-mesh, mach U[0.15,0.25], re U[80,120], "
                                   f"angle U[-2,2] deg, kepes_tecno_roe(minmod), ssprk3 cfl 0.8, t = 0 .. {T}, "
                                   f"forces at {n_out} outputs, QoI window t >= {t_start}",
                       "qois": list(cylinder_names()), "caps_s": {"plain": cap_plain, "batched": cap_batched,
                                                                 "cv": cap_cv}},
            "time_to_rse_measured": r, "clocks": clk.summary(), "impl": "ours",
            "command": "python bench.py --workload cylinder-rse"}


def cylinder_names():
    from tensum_b200 import cylinder
    return cylinder.NAMES


def run_cylinder_rse(args):
    print(json.dumps(cylinder_rse_line(args.final_time, args.outputs, args.t_start, args.seed, args.mc_cap,
                                       args.mc_cap, args.cv_cap)))
    return 0


def run_partitioned(args):
    """The domain-decomposed solve (all partitions on this GPU) against the one-partition step."""
    import torch
    from tensum_b200 import abi, gpu, partition, preproc
    m, prim0 = workload(args)
    g = preproc.preprocess(m)
    parts = [int(x) for x in args.parts.split(",")]
    steps = max(5, min(args.steps, 100))
    V = g.n_vertex
    one, per, seq, ghosts, frontier = {}, {str(n): {} for n in parts}, {str(n): {} for n in parts}, {}, {}
    for flux, recon in args.flux_list:
        P = abi.Problem(g, flux_cfg(flux, recon))
        s = gpu.Solver(P)
        s.set_state(prim0)
        s.step(max(3, args.warmup))
        one[flux] = s.time_phase("step", steps)
        s.close()
        for n in parts:
            for overlap in (True, False):
                ps = partition.PartitionedSolver(P, n, overlap=overlap)
                ps.set_state(prim0)
                ps.step(max(3, args.warmup))
                (per if overlap else seq)[str(n)][flux] = ps.time_steps(steps)
                ghosts[str(n)] = max(p.n_ghost for p in ps.parts) / max(p.n_owned for p in ps.parts)
                frontier[str(n)] = sum(p.n_frontier for p in ps.parts) / sum(p.n_tiles for p in ps.parts)
                ps.close()
        torch.cuda.synchronize()
    nmax = str(max(parts))
    total_ms = sum(per[nmax].values())
    line = {"metric": "vertex-stage updates/s (one mesh in partitions, all on one GPU)",
            "value": len(per[nmax]) * V * 3 / (total_ms / 1e3), "unit": UNIT, "n_gpus": 1, "steps": steps,
            "higher_is_better": True, "dtype": "f64", "data": "synthetic (seeded mesh and field)",
            "config": {"workload": f"kelvin-helmholtz periodic {args.n}x{args.n}, ssprk3 cfl 0.8, fp64, "
                                   f"partitions {args.parts} on one GPU, step captured as one CUDA graph, "
                                   "exchanges overlapped with the interior tiles (and, beside it, not)",
                       "fluxes": [f for f, _ in args.flux_list]},
            "one_partition_ms_per_step": {k: round(v, 4) for k, v in one.items()},
            "partitioned_ms_per_step": {n: {k: round(v, 4) for k, v in d.items()} for n, d in per.items()},
            "partitioned_no_overlap_ms_per_step": {n: {k: round(v, 4) for k, v in d.items()} for n, d in seq.items()},
            "ghost_fraction": {n: round(v, 4) for n, v in ghosts.items()},
            "frontier_tile_fraction": {n: round(v, 4) for n, v in frontier.items()},
            "command": "python bench.py --workload partitioned --parts " + args.parts}
    print(json.dumps(line))
    return 0


def main():
    args = parse()
    if args.workload == "partitioned":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the reference partitions through METIS part files "
                              "and MPI; its single-process run is the single-solve reference arm"}))
            return 0
        return run_partitioned(args)
    if args.workload == "mc":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the reference has no batched ensemble path; its MC "
                              "groups run one sample after another (see the single-solve reference arm)"}))
            return 0
        return run_mc(args)
    if args.workload == "cylinder-rse":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the reference has no batched ensemble path; its MC "
                              "groups run one sample after another (see the single-solve reference arm)"}))
            return 0
        return run_cylinder_rse(args)
    if args.workload == "multilevel":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the reference has no batched ensemble path; its MC "
                              "groups run one sample after another (see the single-solve reference arm)"}))
            return 0
        return run_multilevel(args)
    if args.workload == "cylinder2":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "200k steps of the 131k-vertex Navier-Stokes "
                              "cylinder take about a day on one host core; the single-solve reference arm times "
                              "the reference's own code"}))
            return 0
        return run_cylinder2(args)
    if args.workload == "cylinder":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the reference has no batched ensemble path; its MC "
                              "groups run one sample after another (see the single-solve reference arm)"}))
            return 0
        return run_cylinder(args)
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
