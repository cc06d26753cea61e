"""crava_gpu_posterior_noalloc: the per-bin posterior solve for callers that
cannot allocate device memory (their HBM belongs to their own arena, or they
cannot take the synchronisation of an allocation).  Its scratch is a static
device array inside the library.  Checked through the C ABI against the
regular entry point, crava_gpu_posterior, on two calls in a row (the second
call finds the previous call's tables and counters in the shared scratch).

This file is collected last on purpose."""
import ctypes as C

import numpy as np
import pytest
import torch

from crava_b200 import api, synth

pytestmark = pytest.mark.gpu


def _spectra(ctx, case):
    d = lambda gs: [api.to_device(g) for g in gs]
    mu, data, cov, err = d(case.mu), d(case.data), d(case.cov), d([case.err_corr])[0]
    for g in mu:
        ctx.fft_r2c(g, api.PARAMETER)
    for g in data:
        ctx.fft_r2c(g, api.DATA)
    for g in cov + [err]:
        ctx.fft_r2c(g, api.COVARIANCE)
    torch.cuda.synchronize()
    return mu, data, cov, err


def _clone(grids):
    mu, data, cov, err = grids
    return [g.clone() for g in mu], [g.clone() for g in data], [g.clone() for g in cov], err.clone()


def _rel(a, b):
    a = a.double().cpu().numpy()
    b = b.double().cpu().numpy()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("prec", [api.FP64, api.MIXED])
def test_noalloc_matches_posterior_two_calls(prec):
    case = synth.make_case(32, 24, 64, (0.0, 10.0, 20.0, 30.0, 40.0), 0.1, seed=31)
    ctx = api.Context(case)
    spec = _spectra(ctx, case)
    ref = _clone(spec)
    ctx.posterior(*ref, prec)
    ref_stats = ctx.stats()
    lib = api.load_library()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    for call in range(2):
        out = _clone(spec)
        g = ctx.grids(*out)
        st = api.Stats()
        rc = lib.crava_gpu_posterior_noalloc(C.byref(ctx.params), C.byref(g), prec, stream, C.byref(st))
        assert rc == 0, lib.crava_gpu_status_string(rc)
        assert st.chol_fail_bins == ref_stats.chol_fail_bins
        assert st.nonfinite_bins == 0
        for a, b in zip(out[0] + out[1] + out[2], ref[0] + ref[1] + ref[2]):
            assert _rel(a, b) <= 1e-6


def test_noalloc_rejects_sizes_beyond_its_scratch():
    case = synth.make_case(16, 12, 32, (10.0, 20.0), 0.1, seed=1)
    ctx = api.Context(case)
    p = api.Params.from_buffer_copy(ctx.params)
    p.nzp = 8192
    dummy = torch.zeros(16, device="cuda")
    g = api.Grids()
    for q in range(3):
        g.mu[q] = dummy.data_ptr()
    for l in range(2):
        g.data[l] = dummy.data_ptr()
    for t in range(6):
        g.cov[t] = dummy.data_ptr()
    g.err_corr = dummy.data_ptr()
    lib = api.load_library()
    rc = lib.crava_gpu_posterior_noalloc(C.byref(p), C.byref(g), api.MIXED, None, None)
    assert rc == 7
    assert b"static scratch" in lib.crava_gpu_status_string(rc)
