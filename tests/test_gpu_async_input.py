"""States streamed in while the device steps (tg_set_state_async).

A queued state must become current exactly as tg_set_state makes it (same
bits after the same steps, clocks restarted at its t0), queued states are
taken in order, a refused one leaves the previous state, and the queue holds
two states.  Together with tg_output_begin this is the pipelined path a
caller uses to stream inputs in and results out while the GPU works.
"""
import numpy as np
import pytest

from tensum_b200 import abi, cases, gpu, preproc

pytestmark = pytest.mark.gpu


def _solver(n=65, seed=0):
    m = cases.kh_mesh(n, seed)
    a, phi = cases.kh_coefficients(seed)
    cfg = dict(flux="kepes_tecno_rusanov", reconstruct="minmod",
               boundary={t: ("periodic", {}) for t in (1, 2, 3, 4)}, final_time=1e9, time_stamps=1)
    return gpu.Solver(abi.Problem(preproc.preprocess(m), cfg)), cases.kh_ic(m.coords, a, phi)


def test_queued_states_match_synchronous_ones():
    s, prim0 = _solver()
    ref, _ = _solver()
    ins = [s.output_buffers(False)[0] for _ in range(2)]
    states = [prim0, prim0.copy()]
    states[1][:, 3] *= 1.5                  # another state: scaled v
    for k in range(2):
        ins[k][:] = states[k]
    s.set_state_async(ins[0], 0.0)
    s.set_state_async(ins[1], 0.25)
    out = s.output_buffers(False)[0]
    for k, t0 in enumerate((0.0, 0.25)):
        info = s.step(3)                    # takes the oldest queued state, then steps
        s.output_begin(out)
        s.output_wait()
        ref.set_state(states[k], t0)
        rinfo = ref.step(3)
        assert np.array_equal(out, ref.get_state())
        assert info[0] == rinfo[0] and info[3] == rinfo[3]


def test_refused_state_and_queue_limit():
    s, prim0 = _solver(33)
    s.set_state(prim0)
    s.step(2)
    before = s.get_state()
    buf = s.output_buffers(False)[0]
    buf[:] = prim0
    buf[5, 1] = -1.0                        # p <= 0
    s.set_state_async(buf)
    with pytest.raises(gpu.TensumError) as e:
        s.step(1)
    assert abi.STATUS[e.value.status] == "TG_INVALID_ARG"
    ref, _ = _solver(33)
    ref.set_state(prim0)
    ref.step(3)
    assert np.array_equal(s.get_state(), ref.get_state())   # the step ran on the previous state
    assert not np.array_equal(s.get_state(), before)
    good = [s.output_buffers(False)[0] for _ in range(3)]
    for g in good:
        g[:] = prim0
    s.set_state_async(good[0])
    s.set_state_async(good[1])
    with pytest.raises(gpu.TensumError):
        s.set_state_async(good[2])
    with pytest.raises(gpu.TensumError):
        s.set_state_async(np.ascontiguousarray(prim0))       # pageable memory is refused
    s.set_state(prim0)                                       # drops the queue
    s.step(1)
    ref.set_state(prim0)
    ref.step(1)
    assert np.array_equal(s.get_state(), ref.get_state())
