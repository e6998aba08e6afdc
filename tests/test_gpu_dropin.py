"""The drop-in solver against the stock reference, file for file.

tensum_b200/dropin/_build/tensum_gpu is the reference's own program -- its
command line, parameter and part-file readers, initial conditions from the
parameter file's expressions, sample loop and writers, compiled unchanged --
with FiniteVolume::solve's stage loop (src/fv.cc:2273-2343) replaced by the
C ABI.  Both it and the stock solver built from the same sources
(oracle/_ref/tensum) run the same case directory: a 33 x 33 periodic
isentropic vortex (TeCNO-Roe, minmod, SSP-RK3, CFL 0.8) to t = 0.5 with two
output times, writing the residual log, the global integrals, the solution
files (VTK, with Mach number and vorticity) and the restart file.  The files
must agree: iteration counts exactly, dt, time and the relative residual norm
to 1e-10, the global integrals to their six printed digits, the restart and
solution files to 1e-10 relative L2.
"""
import os
import re
import subprocess

import numpy as np
import pytest

from tensum_b200 import cases
from tensum_b200.mesh import write_part_file
import ref_runner

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DROPIN = os.path.join(ROOT, "tensum_b200", "dropin", "_build", "tensum_gpu")
STOCK = os.path.join(ROOT, "oracle", "_ref", "tensum")

# isentropic vortex of strength 5 in a (1, 1, 1, 1) stream, gas constant 1
VORTEX = {
    "temperature": "1 - 0.4*25/(8*1.4*pi*pi)*exp(1 - x*x - y*y)",
    "xvelocity": "1 - 5/(2*pi)*y*exp(0.5*(1 - x*x - y*y))",
    "yvelocity": "1 + 5/(2*pi)*x*exp(0.5*(1 - x*x - y*y))",
    "zvelocity": "0.0",
    "pressure": "(1 - 0.4*25/(8*1.4*pi*pi)*exp(1 - x*x - y*y))^3.5",
}


def _run(exe, wd):
    r = subprocess.run([exe, "-i", "param.in", "-npart", "1", "-L", "."], cwd=wd, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert "ERROR" not in r.stdout, r.stdout[-2000:]
    out = {}
    for d in sorted(os.listdir(wd)):
        if d.startswith("SAMPLE_"):
            for name in sorted(os.listdir(os.path.join(wd, d))):
                with open(os.path.join(wd, d, name)) as fh:
                    out[name] = fh.read()
    return out


def _numbers(text):
    return [float(t) for t in re.findall(r"[-+]?(?:\d+\.\d*|\.\d+|\d+)(?:[eE][-+]?\d+)?", text)]


@pytest.fixture(scope="module")
def runs(tmp_path_factory):
    for exe in (DROPIN, STOCK):
        assert os.access(exe, os.X_OK), f"{exe} is not built (python -c 'import __graft_entry__ as g; g.build()')"
    m = cases.vortex_mesh(33, seed=5)
    cfg = dict(flux="kepes_tecno_roe", reconstruct="minmod", boundary={t: ("periodic", {}) for t in (1, 2, 3, 4)},
               final_time=0.5, time_stamps=2, cfl=0.8, ic=VORTEX, files=True, variables=["mach", "vorticity"])
    base = tmp_path_factory.mktemp("dropin")
    wd = {}
    for k in ("stock", "gpu"):
        wd[k] = str(base / k)
        os.makedirs(wd[k])
        write_part_file(m, wd[k])
        with open(os.path.join(wd[k], "param.in"), "w") as fh:
            fh.write(ref_runner.param_text(cfg))
    return _run(STOCK, wd["stock"]), _run(DROPIN, wd["gpu"])


def test_same_files(runs):
    stock, gpu = runs
    assert sorted(stock) == sorted(gpu)
    assert "residual.dat" in stock and "global.dat" in stock
    assert any(n.startswith("restart") for n in stock)


def test_residual_log(runs):
    stock, gpu = runs
    a = np.array([_numbers(l) for l in stock["residual.dat"].splitlines() if l.strip()])
    b = np.array([_numbers(l) for l in gpu["residual.dat"].splitlines() if l.strip()])
    assert a.shape == b.shape and a.shape[0] > 10
    assert np.array_equal(a[:, 0], b[:, 0])                       # iterations
    np.testing.assert_allclose(b[:, 1:], a[:, 1:], rtol=1e-10)      # dt, time, relative residual norm


def test_global_integrals(runs):
    stock, gpu = runs
    a = np.array([_numbers(l) for l in stock["global.dat"].splitlines() if l.strip()])
    b = np.array([_numbers(l) for l in gpu["global.dat"].splitlines() if l.strip()])
    assert a.shape == b.shape
    assert np.array_equal(a[:, 0], b[:, 0])
    np.testing.assert_allclose(b[:, 1:], a[:, 1:], rtol=1e-5)       # six printed digits


def test_restart_and_solution_files(runs):
    stock, gpu = runs
    for name in stock:
        if name in ("residual.dat", "global.dat", "time_log.log"):   # the log holds wall times
            continue
        a, b = np.array(_numbers(stock[name])), np.array(_numbers(gpu[name]))
        assert a.shape == b.shape, name
        scale = np.linalg.norm(a)
        if scale == 0.0:                       # e.g. LAST_RESTART_HEAD.txt holds "0"
            assert np.array_equal(a, b), name
            continue
        rel = np.linalg.norm(a - b) / scale
        assert rel <= 1e-10, (name, rel)
