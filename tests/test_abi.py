"""C ABI checks that need no GPU: the in-tree library loads, exports every
function include/crava_gpu.h declares, and rejects bad parameters before
touching a device."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from crava_b200 import api, synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "crava_gpu.h")


def declared():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(crava_gpu_\w+)\s*\(", text)))


def test_header_declares_functions():
    names = declared()
    assert "crava_gpu_create" in names and "crava_gpu_posterior_unit" in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(api.LIB_PATH)
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    assert set(declared()) <= set(api.SYMBOLS)


def test_status_strings():
    lib = api.load_library()
    for code in range(7):
        assert lib.crava_gpu_status_string(code)
    assert lib.crava_gpu_status_string(1).decode() == "invalid argument"


def _params(case, **over):
    wav = np.ascontiguousarray(case.wavelet, np.float32)
    A = np.ascontiguousarray(case.A, np.float32)
    th = np.ascontiguousarray(case.theta_cov, np.float64)
    v0 = np.ascontiguousarray(case.var0, np.float64)
    f = dict(nxp=case.nxp, nyp=case.nyp, nzp=case.nzp, ntheta=case.ntheta, nz=case.nz, precision=1,
             lz=case.lz, min_rel_thick=1.0, low_cut=5.0, high_cut=55.0, wnc=0.1, thickness_mode=0)
    f.update(over)
    p = api.Params(f["nxp"], f["nyp"], f["nzp"], f["ntheta"], f["nz"], f["precision"], f["lz"],
                   f["min_rel_thick"], f["low_cut"], f["high_cut"], f["wnc"], f["thickness_mode"],
                   wav.ctypes.data_as(api.F32P), None, A.ctypes.data_as(api.F32P),
                   th.ctypes.data_as(api.F64P), v0.ctypes.data_as(api.F64P))
    return p, (wav, A, th, v0)


@pytest.mark.parametrize("over", [dict(nxp=11 * 2), dict(nzp=13), dict(ntheta=0), dict(ntheta=9),
                                  dict(precision=7), dict(nz=0), dict(lz=0.0), dict(thickness_mode=2)])
def test_create_rejects_bad_parameters(over):
    case = synth.make_case(16, 12, 32, (10.0, 20.0), 0.1, seed=1)
    p, keep = _params(case, **over)
    lib = api.load_library()
    h = C.c_void_p()
    assert lib.crava_gpu_create(C.byref(p), 0, None, C.byref(h)) == 1
    assert not h.value


def test_null_arguments_rejected():
    lib = api.load_library()
    assert lib.crava_gpu_create(None, 0, None, None) == 1
    assert lib.crava_gpu_fft_r2c(None, None, 1) == 1
    assert lib.crava_gpu_posterior(None, None, 0) == 1
    assert lib.crava_gpu_destroy(None) == 0


def test_create_without_device_reports_nodev():
    """On a machine without a GPU the library reports it instead of failing."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    case = synth.make_case(16, 12, 32, (10.0, 20.0), 0.1, seed=1)
    p, keep = _params(case)
    lib = api.load_library()
    h = C.c_void_p()
    assert lib.crava_gpu_create(C.byref(p), 0, None, C.byref(h)) == 6
