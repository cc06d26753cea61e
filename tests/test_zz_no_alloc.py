"""crava_gpu_posterior_noalloc: the per-bin posterior solve for callers that
cannot allocate device memory (their HBM belongs to their own arena, or they
cannot take the synchronisation of an allocation).  Its scratch is a static
device array inside the library.

Checked through the C ABI against the regular entry point,
crava_gpu_posterior, on two calls in a row with different cases: the second
call has other wavelets, the other thickness mode and a smaller nzp and
ntheta, so it only passes if the call rewrites the tables and counters the
first call left in the shared scratch.  Both calls run the same kernels on
the same inputs as the regular entry point, so the outputs must be equal
bit for bit; device memory in use must not change across the calls.  (The
FP64 form of a context defaults to the Woodbury kernel, whose per-plane
tables live in the context; the allocation-free entry point runs the
square-root kernel, so the regular call it is compared with selects that
kernel, solve_shape 5.)

This file is collected last on purpose."""
import ctypes as C

import numpy as np
import pytest
import torch

from crava_b200 import api, synth

pytestmark = pytest.mark.gpu


def _case_first():
    return synth.make_case(32, 24, 64, (0.0, 10.0, 20.0, 30.0, 40.0), 0.1, seed=31)


def _case_second():
    c = synth.make_case(20, 16, 48, (5.0, 25.0, 45.0), 0.3, seed=32, wavelet_scale_range=(0.8, 1.2),
                        peak_hz=30.0)
    c.thickness_mode = 1
    c.min_rel_thick = 0.8
    return c


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


def _prepare(case, prec):
    """Context, untouched spectra for the allocation-free call, and the
    regular entry point's outputs and stats on the same spectra."""
    ctx = api.Context(case)
    ctx.set_tuning(-1, -1, 0, 2, -1, None, None, 5)
    spec = _spectra(ctx, case)
    ref = _clone(spec)
    ctx.posterior(*ref, prec)
    torch.cuda.synchronize()
    return ctx, _clone(spec), ref, ctx.stats()


def _call(lib, ctx, grids, prec, stream):
    g = ctx.grids(*grids)
    st = api.Stats()
    rc = lib.crava_gpu_posterior_noalloc(C.byref(ctx.params), C.byref(g), prec, stream, C.byref(st))
    assert rc == 0, lib.crava_gpu_status_string(rc)
    return st


@pytest.mark.parametrize("prec", [api.FP64, api.MIXED, api.FP32])
def test_noalloc_matches_posterior_two_calls(prec):
    lib = api.load_library()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    first, second = _case_first(), _case_second()
    assert second.nzp < first.nzp and second.ntheta < first.ntheta
    ctx1, in1, ref1, st1 = _prepare(first, prec)
    ctx2, in2, ref2, st2 = _prepare(second, prec)
    # set-up call (the scratch address of this device; a fresh process
    # loads the array here), on a throw-away copy of the first case
    _call(lib, ctx1, _clone(in1), prec, stream)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    reserved0 = torch.cuda.memory_reserved()
    for ctx, grids, ref, ref_st in ((ctx1, in1, ref1, st1), (ctx2, in2, ref2, st2)):
        st = _call(lib, ctx, grids, prec, stream)
        torch.cuda.synchronize()
        assert st.chol_fail_bins == ref_st.chol_fail_bins
        assert st.nonfinite_bins == ref_st.nonfinite_bins == 0
        for a, b in zip(grids[0] + grids[1] + grids[2], ref[0] + ref[1] + ref[2]):
            assert np.array_equal(a.cpu().numpy(), b.cpu().numpy())
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, "device memory changed across the allocation-free calls"
    assert torch.cuda.memory_reserved() == reserved0


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
    p = api.Params.from_buffer_copy(ctx.params)
    p.nxp = 16384  # the lateral bounds of crava_gpu_create
    rc = lib.crava_gpu_posterior_noalloc(C.byref(p), C.byref(g), api.MIXED, None, None)
    assert rc != 0
