"""Prior and noise covariance grids built on the device
(crava_gpu_fill_prior_cov / crava_gpu_fill_err_corr) against the
restatement of fillInParamCorr / fillInErrCorr, bit for bit, and a
posterior unit fed by them against one fed by uploaded grids."""
import numpy as np
import pytest
import torch

from crava_b200 import api, synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


@pytest.mark.parametrize("shape", [(16, 12, 32), (15, 16, 20), (64, 48, 96)])
@pytest.mark.parametrize("grad", [(0.0, 0.0), (0.3, -0.2), (-1.7, 2.25)])
def test_fills_bitexact(shape, grad):
    nx, ny, nz = shape
    case = synth.make_case(nx, ny, nz, (10.0, 20.0), 0.1, seed=2)
    ctx = api.Context(case)
    cxy = synth.corr_xy(nx, ny, 25.0, 25.0, 500.0)
    circ = api.circ_corr_t(np.exp(-3.0 * (4.0 * np.arange(nz // 2 + 2) / 20.0) ** 2), 1, nz)
    cov = [torch.full_like(api.to_device(case.cov[0]), float("nan")) for _ in range(6)]
    err = torch.full_like(cov[0], float("nan"))
    ctx.fill_prior_cov(cxy, circ, grad[0], grad[1], cov)
    ctx.fill_err_corr(cxy, grad[0], grad[1], err)
    ref = O.fill_prior_cov(nx, ny, nz, cxy, circ, grad[0], grad[1], case.var0)
    for g, r in zip(cov, ref):
        assert np.array_equal(bits(g.cpu().numpy()), bits(r))
    assert np.array_equal(bits(err.cpu().numpy()), bits(O.fill_err_corr(nx, ny, nz, cxy, grad[0], grad[1])))


def test_unit_on_device_filled_prior_equals_uploaded():
    nx, ny, nz = 32, 24, 64
    case = synth.make_case(nx, ny, nz, (0.0, 15.0, 30.0), 0.1, seed=4)
    ctx = api.Context(case, precision=api.FP64)
    d = lambda gs: [api.to_device(g) for g in gs]
    src = (d(case.mu), d(case.data), d(case.cov), d([case.err_corr])[0])
    dev = (d(case.mu), d(case.data), [torch.empty_like(src[2][0]) for _ in range(6)],
           torch.empty_like(src[3]))
    cxy = synth.corr_xy(nx, ny, 25.0, 25.0, 500.0)
    ctx.fill_prior_cov(cxy, synth.circ_corr_t(nz, 4.0, 20.0, 5.0), 0.0, 0.0, dev[2])
    ctx.fill_err_corr(cxy, 0.0, 0.0, dev[3])
    out_a = (d(case.mu), d(case.data), d(case.cov), d([case.err_corr])[0])
    out_b = (d(case.mu), d(case.data), d(case.cov), d([case.err_corr])[0])
    ctx.posterior_unit_oop(src, out_a, api.FP64)
    ctx.posterior_unit_oop(dev, out_b, api.FP64)
    for a, b in zip(out_a[0] + out_a[1] + out_a[2], out_b[0] + out_b[1] + out_b[2]):
        av, bv = a.cpu().numpy()[..., :nx], b.cpu().numpy()[..., :nx]
        assert np.array_equal(av, bv)
