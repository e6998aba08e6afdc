"""Benchmark: vertex-stage updates/s of the FP64 explicit residual/update path.

Workload (one GPU): the Kelvin-Helmholtz shear layer on a seeded, jittered
1025 x 1025 periodic triangulation (1,050,625 stored vertices, 3,147,776
edges), KEPES-TeCNO-Rusanov flux with minmod-limited reconstruction, SSP-RK3,
CFL 0.8, FP64.  A "step" is one SSP-RK3 time step (3 stages) over the whole
mesh; vertex-stage updates per step = 3 x stored vertices.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun each rank runs an independent replica of the solve (the single
solve does not shard: one partition per GPU), so scaling is weak and the value
is the sum over ranks divided by the slowest rank's time.

Keys beyond the base contract:
  roofline      dominant phase (flux pass) against the measured HBM copy peak
  step_roofline whole time step, algorithmic bytes (408 V + 56 E) per stage
  cpu_baseline  the reference's own CPU code on this host (rank 0, N = 1)
  e2e           same metric through the C ABI with host buffers every step
  clocks        SM clock and throttle reasons sampled during the timed region
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


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=1025, help="vertices per side of the periodic mesh")
    ap.add_argument("--flux", default="kepes_tecno_rusanov")
    ap.add_argument("--recon", default="minmod")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--e2e-steps", type=int, default=20)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def workload(args):
    from tensum_b200 import cases
    m = cases.kh_mesh(args.n, seed=args.seed)
    a, phi = cases.kh_coefficients(args.seed)
    prim0 = cases.kh_ic(m.coords, a, phi)
    cfg = dict(flux=args.flux, reconstruct=args.recon, boundary={t: ("periodic", {}) for t in (1, 2, 3, 4)},
               final_time=1.0e9, time_stamps=1, cfl=0.8)
    return m, cfg, prim0


def config_dict(args, m, n_edges):
    return {"workload": f"kelvin-helmholtz periodic {args.n}x{args.n}, {args.flux}+{args.recon}, ssprk3, fp64",
            "mesh_vertices": int(m.n_vertex), "mesh_edges": int(n_edges), "stages_per_step": 3,
            "parallelism": "replicas" if args.gpus > 1 else "single", "l2": "working set > L2 (no flush needed)"}


# ----------------------------------------------------------------------------- clocks
class ClockSampler:
    """Polls NVML (SM clock, throttle reasons) on a thread while the timed region runs."""

    REASONS = {0x1: "gpu_idle", 0x2: "applications_clocks_setting", 0x4: "sw_power_cap", 0x8: "hw_slowdown",
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
                self.reasons |= int(r) & ~0x1
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
def reference_rate(args, m, cfg, prim0, max_steps, warm):
    """Time the reference's own CPU code (oracle/_ref harness) on the same workload."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_runner
    if not ref_runner.harness_available():
        return None
    steps = warm + max_steps
    with tempfile.TemporaryDirectory(prefix="tensum_ref_bench_") as wd:
        d = ref_runner.run_case(m, cfg, prim0, steps, 0, workdir=wd, timeout=3600)
    st = d["step_s"][warm:]
    sec = float(np.sum(st))
    rate = m.n_vertex * 3 * len(st) / sec
    return {"value": rate, "unit": UNIT, "cores": 1, "kind": "reference",
            "sample": f"{len(st)} SSP-RK3 steps of the full {args.n}x{args.n} workload after {warm} warm-up "
                      f"step(s); reference sources built -O3 with a serial MPI stub (one process, one core)",
            "seconds": sec}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    m, cfg, prim0 = workload(args)
    steps = max(1, min(args.steps, 3))
    warm = 1 if args.warmup > 0 else 0
    r = reference_rate(args, m, cfg, prim0, steps, warm)
    from tensum_b200 import preproc
    ne = preproc.preprocess(m).n_face
    if r is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/tensum_harness not built on this host"}))
        return 0
    line = {"metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": args.gpus, "steps": steps,
            "warmup": warm, "ms_per_step": 1e3 * r["seconds"] / steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded mesh and field)",
            "config": config_dict(args, m, ne), "impl": "reference",
            "cpu_baseline": {k: r[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": r["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ----------------------------------------------------------------------------- our arm
def traffic_from_profile(kernel_tag):
    """Per-launch DRAM bytes of the dominant phase from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", f"{kernel_tag}.txt")
    try:
        for line in open(p):
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
    m, cfg, prim0 = workload(args)
    g = preproc.preprocess(m)
    P = abi.Problem(g, cfg)
    s = gpu.Solver(P)
    s.set_state(prim0)
    V, E = g.n_vertex, g.n_face
    stream = torch.cuda.ExternalStream(s.stream_ptr())

    s.step(max(3, args.warmup))
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev) as clk:
        torch.cuda.synchronize()
        ev0.record(stream)
        info = s.step(args.steps)
        ev1.record(stream)
        torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    if dist:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    vs = V * 3 * args.steps * world
    value = vs / (ms / 1e3)
    ms_step = ms / args.steps
    launches_step = int(s.query("kernels_per_step"))

    # roofline of the dominant phase (flux pass) and of the whole step
    peak, peak_kind = measured_peaks()
    flux_ms = s.time_phase("flux", 50)
    flux_bytes = 144 * V + 24 * E            # U 32V + grad 64V + coords 16V + edges 24E + R 32V
    step_bytes = 3 * (408 * V + 56 * E)
    grad_ms = s.time_phase("gradient", 50)
    upd_ms = s.time_phase("update", 50)
    dt_ms = s.time_phase("dt", 50)
    roof = {"bound": "hbm", "kernel": "flux pass (edge flux + residual assembly)",
            "achieved": flux_bytes / (flux_ms / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
            "frac": flux_bytes / (flux_ms / 1e3) / 1e9 / peak, "traffic": traffic_from_profile("flux_pass_kh1025"),
            "algorithmic_bytes_per_launch": flux_bytes, "ms_per_launch": flux_ms, "peak_source": peak_kind}
    step_roof = {"achieved": step_bytes / (ms_step / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                 "frac": step_bytes / (ms_step / 1e3) / 1e9 / peak, "bytes_per_step": step_bytes,
                 "phase_ms": {"gradient": grad_ms, "flux": flux_ms, "update": upd_ms, "dt": dt_ms}}

    # end to end through the C ABI with host buffers every step
    s.set_state(prim0)
    host_out = np.empty((V, 5))
    ne2e = max(1, min(args.e2e_steps, args.steps))
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(ne2e):
        s.set_state(prim0)
        s.step(1)
        host_out[:] = s.get_state()
    e2e_s = time.perf_counter() - t0
    if dist:
        t = torch.tensor([e2e_s], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e = {"value": V * 3 * ne2e * world / e2e_s, "unit": UNIT, "h2d_bytes_per_step": 32 * V,
           "d2h_bytes_per_step": 32 * V, "steps": ne2e,
           "path": "tg_set_state(host AoS) + tg_step(1) + tg_get_state(host AoS) per step"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        r = reference_rate(args, m, cfg, prim0, 2, 1)
        if r is not None:
            cpu = {k: r[k] for k in ("value", "unit", "cores", "kind", "sample")}

    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": max(3, args.warmup), "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded mesh and field)",
            "config": config_dict(args, m, E), "roofline": roof, "step_roofline": step_roof, "cpu_baseline": cpu,
            "e2e": e2e, "gpu_launches": launches_step * args.steps, "clocks": clk.summary(),
            "sim_time": info[0], "impl": "ours"}
    print(json.dumps(line))
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
