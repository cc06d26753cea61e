"""Parity at the headline size and at the uneven vintage grids.

Headline: 256x256x512, 5 angles at 0/10/20/30/40 degrees, wavelet scales
U[0.8, 1.2], noise at 10 % and 30 % of the signal energy (the full-size
plain configuration).  Vintages: 96x200x300 and 192x160x384, 5 angles
(the uneven grids of the batched configuration).

* FP32 form (the reference's float arithmetic and operation order), the
  whole unit on the real grids, against the reference's own numerics
  (oracle/_ref: FFTW 2.1.2 and lib_matr.c in the restated loop of
  src/crava.cpp:1042-1151): relative L2 error per output < 2e-5.
* FP64 and mixed forms, the per-bin solve on identical spectra (the
  device's forward transforms, downloaded), against the FP64 oracle:
  relative L2 error per output < 1e-6 (FP64) and < 1e-5 (mixed), and the
  same failed-bin count.

Each case is built once per module (about 25 s of host time at the
headline size); the reference unit takes about 15 s of one core.
"""
import numpy as np
import pytest
import torch

from crava_b200 import api, synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu

ANGLES5 = (0.0, 10.0, 20.0, 30.0, 40.0)
_CASES = {}


def _case(name):
    if name not in _CASES:
        if name == "full10":
            _CASES[name] = synth.config_full(seed=2, noise_frac=0.10)
        elif name == "full30":
            _CASES[name] = synth.config_full(seed=2, noise_frac=0.30)
        elif name == "v96x200x300":
            _CASES[name] = synth.make_case(96, 200, 300, ANGLES5, 0.10, seed=43, wavelet_scale_range=(0.8, 1.2))
        elif name == "v192x160x384":
            _CASES[name] = synth.make_case(192, 160, 384, ANGLES5, 0.10, seed=44, wavelet_scale_range=(0.8, 1.2))
        else:
            raise KeyError(name)
    return _CASES[name]


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


CASES = ["full10", "full30", "v96x200x300", "v192x160x384"]


@pytest.mark.parametrize("name", CASES)
def test_fp32_unit_vs_reference(name):
    assert O.have_ref(), "oracle/_ref (the reference's FFTW 2.1.2 and lib_matr.c) is not built"
    case = _case(name)
    ctx = api.Context(case)
    d = lambda gs: [api.to_device(g) for g in gs]
    mu, data, cov, err = d(case.mu), d(case.data), d(case.cov), d([case.err_corr])[0]
    ctx.posterior_unit(mu, data, cov, err, api.FP32)
    st = ctx.stats()
    omu, ores, ocov, ofail = O.unit_fp32(case, "ref")
    assert st.chol_fail_bins == ofail
    assert st.nonfinite_bins == 0
    nx = case.nxp
    worst = 0.0
    for g, o in zip(mu + data + cov, omu + ores + ocov):
        e = _rel(g.cpu().numpy()[..., :nx].astype(np.float64), o[..., :nx].astype(np.float64))
        worst = max(worst, e)
        assert e < 2e-5, e
    print(f"{name}: FP32 unit vs reference, worst output rel L2 {worst:.2e}")


@pytest.mark.parametrize("name", CASES)
def test_fp64_and_mixed_solve_vs_fp64_oracle(name):
    case = _case(name)
    ctx = api.Context(case)
    d = lambda gs: [api.to_device(g) for g in gs]
    mu, data, cov, err = d(case.mu), d(case.data), d(case.cov), d([case.err_corr])[0]
    for g in mu:
        ctx.fft_r2c(g, api.PARAMETER)
    for g in data:
        ctx.fft_r2c(g, api.DATA)
    for g in cov + [err]:
        ctx.fft_r2c(g, api.COVARIANCE)
    torch.cuda.synchronize()
    host = lambda gs: [g.cpu().numpy() for g in gs]
    sp = {"mu": host(mu), "data": host(data), "cov": host(cov), "err": err.cpu().numpy()}
    omu, ores, ocov, ofail = O.posterior_fp64(case, sp)
    ref = omu + ores + ocov
    ctx.set_kz_tables(O.kz_tables(case, "orc"))  # the oracle's tables: the solve alone is compared
    for prec, bar in ((api.FP64, 1e-6), (api.MIXED, 1e-5)):
        m, dd, c = [g.clone() for g in mu], [g.clone() for g in data], [g.clone() for g in cov]
        ctx.posterior(m, dd, c, err, prec)
        st = ctx.stats()
        assert st.chol_fail_bins == ofail
        assert st.nonfinite_bins == 0
        worst = 0.0
        for g, o in zip(m + dd + c, ref):
            e = _rel(api.complex_view(g.cpu().numpy(), case.nxp).astype(np.complex128), o)
            worst = max(worst, e)
            assert e < bar, (prec, e)
        print(f"{name}: {'FP64' if prec == api.FP64 else 'mixed'} solve vs FP64 oracle, "
              f"worst output rel L2 {worst:.2e}")
