"""The C-ABI library loads and exports every entry point the header declares."""
import ctypes as C
import os
import re

import pytest

from tensum_b200 import build, gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "tensum_gpu.h")).read()
    return sorted(set(re.findall(r"^\s*(?:tg_status|const char\*|int)\s+(tg_\w+)\s*\(", text, re.M)))


def test_header_declares_the_hot_path():
    syms = declared_symbols()
    for s in ["tg_create", "tg_destroy", "tg_set_state", "tg_get_state", "tg_compute_dt", "tg_gradients",
              "tg_residual", "tg_update", "tg_residual_norm", "tg_step", "tg_global"]:
        assert s in syms


def test_library_exports_every_declared_symbol():
    build.build()
    lib = C.CDLL(gpu.LIB_PATH)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_abi_version():
    lib = gpu.load()
    assert lib.tg_abi_version() == gpu.ABI_VERSION == 4


@pytest.mark.skipif(gpu.load() is None, reason="library not loadable")
def test_create_without_device_reports_no_device():
    """On a host without a GPU the path refuses to run instead of falling back."""
    from tests.conftest import cuda_device_present
    if cuda_device_present():
        pytest.skip("a CUDA device is present")
    from tensum_b200 import abi, cases, preproc
    m = cases.vortex_mesh(9, 0)
    P = abi.Problem(preproc.preprocess(m), dict(boundary={t: ("periodic", {}) for t in (1, 2, 3, 4)}))
    with pytest.raises(gpu.TensumError) as e:
        gpu.Solver(P)
    assert e.value.status == 6
