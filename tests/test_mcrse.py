"""Host logic of the time-to-RSE Monte Carlo arms (tensum_b200/mcrse.py) with
stand-in solvers of known distribution, on the CPU: the stopping rule, the cap
and its 1/sqrt(N) extrapolation, and the summary's speed-ups, including the
plain-MC time from the sample count over the control-variate arm's samples."""
import time

import numpy as np
import pytest

from tensum_b200 import cv, mcrse


class _Stub:
    def close(self):
        pass


def _draw(i):
    # QoIs with relative spreads of 10% and 30% around 1 and 2
    r = np.random.default_rng(1000 + i)
    return np.array([1.0 + 0.1 * r.standard_normal(), 2.0 + 0.6 * r.standard_normal()])


def test_plain_arm_stops_at_target_in_draw_order():
    out = mcrse.plain_arm(_Stub, lambda s, i: _draw(i), rse=0.02, handles=4, cap_s=60.0, check_every=32,
                          min_samples=64)
    assert out["reached"]
    assert max(out["rse_mean"]) <= 0.02 and max(out["rse_var"]) <= 0.02
    # the estimate was made on the first `samples` draws, in order
    Y = np.stack([_draw(i) for i in range(out["samples"])])
    rm, rv = cv.rse_now(Y)
    assert np.allclose(rm, out["rse_mean"]) and np.allclose(rv, out["rse_var"])


def test_plain_arm_cap_extrapolates_by_inverse_square_root():
    def slow(s, i):
        time.sleep(0.002)
        return _draw(i)
    out = mcrse.plain_arm(_Stub, slow, rse=1e-4, handles=2, cap_s=0.5, check_every=16, min_samples=32)
    assert not out["reached"]
    worst = max(max(out["rse_mean"]), max(out["rse_var"]))
    assert out["extrapolated_wall_s"] == pytest.approx(out["wall_s"] * (worst / 1e-4) ** 2)


def test_batched_arm_stops_at_first_batch_meeting_target():
    def run_batch(start, n):
        X = np.zeros((n, 1))
        return X, np.stack([_draw(start + s) for s in range(n)])
    out = mcrse.batched_arm(run_batch, rse=0.02, batch_n=256)
    assert out["reached"] and out["samples"] == out["batches"] * 256
    Y = np.stack([_draw(i) for i in range(out["samples"] - 256)])
    rm, rv = cv.rse_now(Y)
    assert max(rm.max(), rv.max()) > 0.02        # one batch fewer would not have reached it


def test_summary_speedups_and_sample_count_estimate():
    pl = dict(wall_s=120.0, samples=100, reached=False, extrapolated_wall_s=1000.0)
    bt = dict(wall_s=50.0, reached=True)
    cvr = dict(wall_s=80.0, reached=True, samples=4000, plain_rse_mean_same_samples=[0.002, 0.003],
               plain_rse_var_same_samples=[0.02, 0.015])
    s = mcrse._summary(0.01, pl, bt, cvr)
    assert s["speedup_batched_vs_plain_fp64"] == pytest.approx(1000.0 / 50.0)
    assert s["speedup_cv_vs_plain_fp64"] == pytest.approx(1000.0 / 80.0)
    by = s["plain_fp64_by_sample_count"]
    assert by["samples_needed"] == pytest.approx(4000 * 4.0)          # worst 0.02 against 0.01
    assert by["wall_s"] == pytest.approx(16000 * 1.2)                  # 120 s / 100 samples each
    assert s["speedup_cv_vs_plain_fp64_by_sample_count"] == pytest.approx(19200.0 / 80.0)
    assert s["time_kind"] == {"plain_fp64": "extrapolated from a capped run", "batched_fp32": "measured",
                              "batched_fp32_cv": "measured"}
