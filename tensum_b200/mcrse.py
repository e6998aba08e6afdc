"""Measured wall time to a target relative standard error, three Monte Carlo arms.

Each arm draws the same sequence of samples and stops as soon as the relative
standard errors of the mean AND of the variance estimate of every QoI are at
or below the target (cv.rse_now); the wall clock runs from the first sample to
that point and includes everything a user pays per sample: initial condition,
solve, QoI, and for the surrogate arm its training solves, training and
evaluations.  Handle and batch creation are set-up and stay outside.

  plain FP64 MC   the FP64 solver, `handles` handles stepping at once (one
                  host thread each); the estimate uses the samples completed
                  in draw order
  batched FP32 MC batches of `batch_n` samples in one FP32 ensemble launch
  FP32 + CV       n_train batched solves train the surrogate; evaluation
                  batches follow, each paired with the surrogate at its
                  inputs, plus 2^20 surrogate evaluations at fresh inputs;
                  the control-variate estimator (plain MC where it does not help)

An arm may have a wall-clock cap; an arm that hits it reports the errors it
reached and the time the 1/sqrt(N) law gives for the target from its measured
rate, marked as extrapolated.  Because a capped plain arm may hold few samples
(the error of a variance estimate is itself noisy there), the summary adds a
second plain time: the sample count the plain estimator needs, judged on all
the control-variate arm's solver samples, times the plain arm's measured wall
time per sample.

Two workloads: Kelvin-Helmholtz samples (rnd-file rows; QoIs 0.5 rho v^2,
0.5 rho u^2 and -rho s/(gamma-1) integrated over the mesh at the output time)
and the Navier-Stokes cylinder with uncertain Mach, Re and inflow angle (QoIs
of tensum_b200.cylinder over the force history).
"""
from __future__ import annotations

import threading
import time

import numpy as np

from . import abi, batch, cases, cv, cylinder, gpu, mlp


def _done(y, rse, g=None, ge=None):
    rm, rv = cv.rse_now(y, g, ge)
    return bool(np.all(rm <= rse) and np.all(rv <= rse)), rm, rv


def _capped(out, rm, rv, rse, cap_s):
    worst = max(float(np.max(rm)), float(np.max(rv)))
    out["extrapolated_wall_s"] = out["wall_s"] * (worst / rse) ** 2
    out["note"] = f"cap of {cap_s:g} s reached; extrapolated_wall_s follows the 1/sqrt(N) law"
    return out


def plain_arm(make_solver, solve_one, rse, handles=8, cap_s=120.0, check_every=64, min_samples=64):
    """solve_one(solver, i) -> QoI vector of sample i on an FP64 handle."""
    solvers = [make_solver() for _ in range(handles)]
    ys, lock, stop, errors = {}, threading.Lock(), threading.Event(), []
    counter = iter(range(1 << 40))

    def work(k):
        try:
            while not stop.is_set():
                with lock:
                    i = next(counter)
                y = solve_one(solvers[k], i)
                with lock:
                    ys[i] = y
        except Exception as e:          # re-raised on the calling thread
            errors.append(e)
            stop.set()

    th = [threading.Thread(target=work, args=(k,)) for k in range(handles)]
    t0 = time.perf_counter()
    for t in th:
        t.start()
    n_checked, reached, rm, rv = 0, False, None, None
    while not stop.is_set():
        time.sleep(0.05)
        with lock:
            n = 0
            while n in ys:
                n += 1
        if n >= max(min_samples, n_checked + check_every):
            n_checked = n
            with lock:
                Y = np.stack([ys[i] for i in range(n)])
            reached, rm, rv = _done(Y, rse)
            if reached:
                break
        if time.perf_counter() - t0 > cap_s and rm is not None:
            break
    wall = time.perf_counter() - t0
    stop.set()
    for t in th:
        t.join()
    for s in solvers:
        s.close()
    if errors:
        raise errors[0]
    out = dict(wall_s=wall, samples=n_checked, reached=reached, handles=handles,
               rse_mean=rm.tolist(), rse_var=rv.tolist())
    return out if reached else _capped(out, rm, rv, rse, cap_s)


def batched_arm(run_batch, rse, batch_n, cap_s=float("inf"), max_batches=64):
    """run_batch(start, n) -> (X, QoIs) of samples start .. start + n - 1, one batched launch."""
    Y = []
    t0 = time.perf_counter()
    for k in range(max_batches):
        Y.append(run_batch(k * batch_n, batch_n)[1])
        reached, rm, rv = _done(np.concatenate(Y), rse)
        if reached or time.perf_counter() - t0 > cap_s:
            break
    wall = time.perf_counter() - t0
    out = dict(wall_s=wall, samples=len(Y) * batch_n, batches=len(Y), batch=batch_n, reached=reached,
               rse_mean=rm.tolist(), rse_var=rv.tolist())
    return out if reached else _capped(out, rm, rv, rse, cap_s)


def cv_arm(run_batch, draw_extra, rse, n_train, batch_n, train_batch=None, n_extra=1 << 20, epochs=300, mb=128,
           lr=2e-3, cap_s=float("inf"), max_batches=64):
    """Surrogate trained on the first n_train solves, then evaluation batches with
    the control-variate estimator; draw_extra(n) -> n fresh inputs."""
    t0 = time.perf_counter()
    tb = train_batch or batch_n
    Xtr, Ytr = [], []
    for k in range(0, n_train, tb):
        X, Y = run_batch(k, min(tb, n_train - k))
        Xtr.append(X)
        Ytr.append(Y)
    Xtr, Ytr = np.concatenate(Xtr), np.concatenate(Ytr)
    net = mlp.MLP(Xtr.shape[1], Ytr.shape[1], seed=1)
    net.fit(Xtr, Ytr, epochs=epochs, batch=mb, lr=lr)
    t_train = time.perf_counter() - t0
    g_extra = net.predict(draw_extra(n_extra), precision=1)
    Y, G = [], []
    for k in range(max_batches):
        X, y = run_batch(n_train + k * batch_n, batch_n)
        Y.append(y)
        G.append(net.predict(X, precision=1))
        reached, rm, rv = _done(np.concatenate(Y), rse, np.concatenate(G), g_extra)
        if reached or time.perf_counter() - t0 > cap_s:
            break
    wall = time.perf_counter() - t0
    est = cv.estimate(np.concatenate(Y), np.concatenate(G), g_extra)
    # the plain estimator's errors on every solver sample this arm drew (training ones included)
    pm, pv = cv.rse_now(np.concatenate([Ytr] + Y))
    out = dict(wall_s=wall, train_s=t_train, samples=n_train + len(Y) * batch_n, train_samples=n_train,
               eval_samples=len(Y) * batch_n, surrogate_evals=n_extra, reached=reached,
               rse_mean=rm.tolist(), rse_var=rv.tolist(), gain=[float(x) for x in est["gain"]],
               used=[bool(x) for x in est["used"]], plain_rse_mean_same_samples=pm.tolist(),
               plain_rse_var_same_samples=pv.tolist())
    return out if reached else _capped(out, rm, rv, rse, cap_s)


def _summary(rse, pl, bt, cvr):
    def t(a):
        return a["wall_s"] if a["reached"] else a["extrapolated_wall_s"]
    # A second plain-MC time that does not lean on the capped arm's few samples: the plain
    # estimator's errors over the control-variate arm's (many more) solver samples give the
    # sample count it needs, times the plain arm's measured wall time per sample.
    worst = max(max(m, v) for m, v in zip(cvr["plain_rse_mean_same_samples"], cvr["plain_rse_var_same_samples"]))
    need = cvr["samples"] * (worst / rse) ** 2
    per = pl["wall_s"] / max(pl["samples"], 1)
    by_count = {"samples_needed": need, "wall_s_per_sample": per, "wall_s": need * per,
                "from": f"plain estimator errors over the {cvr['samples']} solver samples of the control-variate arm"}
    return {"rse": rse, "targets": "mean and variance of every QoI", "plain_fp64": pl, "batched_fp32": bt,
            "batched_fp32_cv": cvr, "speedup_batched_vs_plain_fp64": t(pl) / t(bt),
            "speedup_cv_vs_plain_fp64": t(pl) / t(cvr),
            "plain_fp64_by_sample_count": by_count,
            "speedup_cv_vs_plain_fp64_by_sample_count": by_count["wall_s"] / t(cvr),
            "speedup_batched_vs_plain_fp64_by_sample_count": by_count["wall_s"] / t(bt),
            "time_kind": {k: ("measured" if a["reached"] else "extrapolated from a capped run")
                          for k, a in (("plain_fp64", pl), ("batched_fp32", bt), ("batched_fp32_cv", cvr))}}


# ------------------------------------------------------------ Kelvin-Helmholtz
def _kh_qoi(q: np.ndarray, aw: np.ndarray, gamma: float = 1.4) -> np.ndarray:
    rho = q[:, 1] / q[:, 0]
    ent = np.log(q[:, 1]) - gamma * np.log(rho)
    return np.array([np.sum(0.5 * rho * q[:, 3] ** 2 * aw), np.sum(0.5 * rho * q[:, 2] ** 2 * aw),
                     np.sum(-rho * ent / (gamma - 1.0) * aw)])


def measure(g, m, cfg, rows_of, rse=0.01, handles=8, cap_s=120.0, batch_n=1024, n_train=1024, seed=0) -> dict:
    """Kelvin-Helmholtz samples from rnd rows (initial conditions from the
    parameter file's expressions with pert(4, ...) on the device for the FP64
    handles, generated by the batch for the ensembles)."""
    P = abi.Problem(g, cfg)
    w = np.ones(m.n_vertex)
    for st in m.periodic_sets:
        w[st] = 1.0 / len(st)
    aw = g.dcarea * w
    b = batch.Batch([(P, batch_n)])

    def run_batch(start, n):
        X = np.stack([rows_of(start + s) for s in range(batch_n)])
        b.set_kh(0, X)
        b.advance(1)
        return X[:n], b.integrals(0)[:n]

    def make_solver():
        s = gpu.Solver(P)
        s.fields = gpu.expr_fields(cases.kh_expressions())   # per handle: each holds its rnd row
        return s

    def solve_one(s, i):
        s.set_state_expr(s.fields, rnd=rows_of(i))
        s.advance(1)
        return _kh_qoi(s.get_state(), aw)

    bt = batched_arm(run_batch, rse, batch_n)
    cvr = cv_arm(run_batch, lambda n: np.random.default_rng(10 ** 7 + seed).uniform(0.0, 1.0, size=(n, 20)),
                 rse, n_train, batch_n)
    pl = plain_arm(make_solver, solve_one, rse, handles, cap_s)
    return _summary(rse, pl, bt, cvr)


# ------------------------------------------------------------ cylinder
def measure_cylinder(g, coords, T, n_out, t_start, rse=0.01, seed=0, handles=8, batch_n=512, n_train=256,
                     cap_plain_s=180.0, cap_batched_s=180.0, cap_cv_s=float("inf")) -> dict:
    """The Navier-Stokes cylinder over uncertain (Mach, Re, angle): every sample
    runs t = 0 .. T with the wall force at n_out outputs, QoIs over t >= t_start."""
    X_all = cylinder.draw_inputs(1 << 16, seed)
    cfgs = {}

    def cfg_of(i):
        if i not in cfgs:
            mach, re, ang = X_all[i]
            cfgs[i] = cases.cylinder_config(mach, re, ang, T, n_out)
        return cfgs[i]

    def run_batch(start, n):
        X = X_all[start:start + n]
        r = cylinder.run_batched(g, coords, X, T, n_out, t_start, tune=False)
        return X, r["y"]

    P0 = abi.Problem(g, cfg_of(0))

    def solve_one(s, i):
        mach, _, ang = X_all[i]
        s.update_parameters(abi.Problem(g, cfg_of(i)))
        s.set_state(cases.cylinder_ic(coords, mach, ang))
        hist = [s.forces(cylinder.FORCES)[0]]
        for k in range(1, n_out + 1):
            s.advance(k)
            hist.append(s.forces(cylinder.FORCES)[0])
        return cylinder.qois(np.linspace(0.0, T, n_out + 1), np.array(hist), mach, ang, t_start)

    bt = batched_arm(run_batch, rse, batch_n, cap_s=cap_batched_s)
    cvr = cv_arm(run_batch, lambda n: cylinder.draw_inputs(n, 10 ** 7 + seed), rse, n_train, batch_n,
                 train_batch=n_train, epochs=400, mb=64, cap_s=cap_cv_s)
    pl = plain_arm(lambda: gpu.Solver(P0), solve_one, rse, handles, cap_plain_s, check_every=16, min_samples=32)
    return _summary(rse, pl, bt, cvr)
