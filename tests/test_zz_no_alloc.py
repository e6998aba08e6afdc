"""The allocation-free residual-norm entry point agrees with the handle-based one.

tg_residual_norm_noalloc serves callers that cannot allocate device memory
while they run (hosts that reserve all GPU memory up front, code that runs
while a CUDA graph is being captured elsewhere, real-time loops): it reads
caller-owned device buffers and keeps its partial sums in a fixed device
array inside the library.  This test feeds it the residual of a real solve,
in the reference's Flux layout, and compares it with tg_residual_norm of the
same handle within the tolerance the parity tests use (1e-12 relative), on two
calls in a row (the second call reuses the shared scratch array left by the
first).  The file is named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

from tests.helpers import rel_l2
from tensum_b200 import abi, cases, gpu, preproc

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _setup(n, seed, flux, recon):
    m = cases.kh_mesh(n, seed)
    a, phi = cases.kh_coefficients(seed)
    prim0 = cases.kh_ic(m.coords, a, phi)
    cfg = dict(flux=flux, reconstruct=recon, boundary={t: ("periodic", {}) for t in (1, 2, 3, 4)},
               final_time=1e9, time_stamps=1)
    g = preproc.preprocess(m)
    s = gpu.Solver(abi.Problem(g, cfg))
    s.set_state(prim0)
    w = np.ones(m.n_vertex)
    for st in m.periodic_sets:
        w[st] = 1.0 / len(st)
    return s, g, w


def _noalloc(lib, res, area, w, total0):
    import torch
    dev = torch.device("cuda")
    r = torch.from_numpy(np.ascontiguousarray(res, np.float64)).to(dev)
    a = torch.from_numpy(np.ascontiguousarray(area, np.float64)).to(dev)
    ww = torch.from_numpy(np.ascontiguousarray(w, np.float64)).to(dev)
    out = torch.full((6,), float("nan"), dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    st = lib.tg_residual_norm_noalloc(C.c_void_p(r.data_ptr()), C.c_void_p(a.data_ptr()), C.c_void_p(ww.data_ptr()),
                                      int(res.shape[0]), float(total0), C.c_void_p(out.data_ptr()), None)
    assert st == 0, lib.tg_noalloc_last_error().decode()
    torch.cuda.synchronize()
    return out.cpu().numpy()


def test_noalloc_norm_matches_handle_norm_twice():
    lib = gpu.load()
    lib.tg_residual_norm_noalloc.argtypes = [C.c_void_p] * 3 + [C.c_int, C.c_double, C.c_void_p, C.c_void_p]
    lib.tg_residual_norm_noalloc.restype = C.c_int
    lib.tg_noalloc_last_error.restype = C.c_char_p
    s, g, w = _setup(129, 3, "kepes_tecno_rusanov", "minmod")
    # first call: iteration 0 sets the normaliser
    res = s.residual()
    ref0 = s.residual_norm(0)
    got0 = _noalloc(lib, res, g.dcarea, w, 0.0)
    assert rel_l2(got0, ref0) <= TOL
    # second call in a row, on a later residual; normalised like the handle's
    # (its normaliser was reset by the first step of tg_step)
    s.step(3)
    res = s.residual()
    ref1 = s.residual_norm(5)
    got1 = _noalloc(lib, res, g.dcarea, w, ref1[5])
    assert rel_l2(got1, ref1) <= TOL
    assert got1[5] == ref1[5]


def test_noalloc_rejects_oversized_input():
    lib = gpu.load()
    lib.tg_residual_norm_noalloc.argtypes = [C.c_void_p] * 3 + [C.c_int, C.c_double, C.c_void_p, C.c_void_p]
    lib.tg_residual_norm_noalloc.restype = C.c_int
    lib.tg_noalloc_last_error.restype = C.c_char_p
    import torch
    t = torch.zeros(8, dtype=torch.float64, device="cuda")
    p = C.c_void_p(t.data_ptr())
    st = lib.tg_residual_norm_noalloc(p, p, p, 268435456 + 1, 0.0, p, None)
    assert st == 4
    assert b"TG_NOALLOC_MAX_VERTICES" in lib.tg_noalloc_last_error()


def _bind():
    lib = gpu.load()
    lib.tg_residual_norm_noalloc.argtypes = [C.c_void_p] * 3 + [C.c_int, C.c_double, C.c_void_p, C.c_void_p]
    lib.tg_residual_norm_noalloc.restype = C.c_int
    lib.tg_noalloc_last_error.restype = C.c_char_p
    return lib


def test_noalloc_strided_blocks_match_numpy():
    """Above 2048 blocks x 256 threads (524,288 vertices) the grid is capped and
    every thread strides over several vertices: compare with the formula in numpy."""
    lib = _bind()
    nv = 900_001
    rng = np.random.default_rng(7)
    res = rng.standard_normal((nv, 5))
    area = rng.uniform(0.5, 2.0, nv)
    w = np.where(rng.uniform(size=nv) < 0.01, 0.5, 1.0)
    q = res[:, [0, 1, 2, 4]] / area[:, None]
    n = np.sqrt((q * q * w[:, None]).sum(axis=0)) / nv
    total = np.sqrt(n[0] ** 2 + (n[1] ** 2 + n[2] ** 2 + 0.0) + n[3] ** 2)
    for _ in range(2):
        got = _noalloc(lib, res, area, w, 0.0)
        assert rel_l2(got[:4], n) <= TOL
        assert abs(got[5] - total) <= TOL * total and got[4] == 1.0


def test_noalloc_zero_residual_and_null_buffer():
    lib = _bind()
    nv = 1000
    got = _noalloc(lib, np.zeros((nv, 5)), np.ones(nv), np.ones(nv), 0.0)
    # a zero first-iteration total makes the normaliser 1 (src/fv.cc:1860-1873)
    assert got[5] == 1.0 and got[4] == 0.0 and np.all(got[:4] == 0.0)
    import torch
    t = torch.zeros(8, dtype=torch.float64, device="cuda")
    p = C.c_void_p(t.data_ptr())
    assert lib.tg_residual_norm_noalloc(None, p, p, 4, 0.0, p, None) == 4
    assert lib.tg_residual_norm_noalloc(p, p, p, 4, 0.0, None, None) == 4
    assert b"NULL" in lib.tg_noalloc_last_error()
