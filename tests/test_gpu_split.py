"""A grid split over GPUs, its device half on one GPU: the x/y-only and
z-only transforms equal the 3-D transform bit for bit, and the split unit
(slab and column-shard contexts, the exchange degenerate for one rank)
equals the one-GPU posterior unit bit for bit.  The exchange itself is
tested with gloo ranks on CPU (test_dist_gloo.py)."""
import numpy as np
import pytest
import torch

from crava_b200 import api, dist_grid as G, synth

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("shape", [(64, 48, 96), (15, 16, 20)])
@pytest.mark.parametrize("gtype", [api.DATA, api.COVARIANCE, api.PARAMETER])
def test_xy_and_z_passes_are_the_3d_transform(shape, gtype):
    case = synth.make_case(*shape, (10.0, 20.0), 0.1, seed=6)
    ctx = api.Context(case)
    g = case.data[0] if gtype != api.COVARIANCE else case.cov[1]
    a, b = api.to_device(g), api.to_device(g)
    ctx.fft_r2c(a, gtype)
    ctx.fft_xy(b, -1, gtype)
    ctx.fft_z(b, -1)
    assert torch.equal(a, b)
    ctx.fft_c2r(a, gtype)
    ctx.fft_z(b, 1)
    ctx.fft_xy(b, 1, gtype)
    nx = shape[0]
    assert torch.equal(a[..., :nx], b[..., :nx])


@pytest.mark.parametrize("precision", [api.FP64, api.MIXED])
def test_split_unit_one_rank_equals_unit(precision):
    case = synth.make_case(32, 24, 64, (0.0, 10.0, 20.0, 30.0, 40.0), 0.1, seed=12)
    ctx = api.Context(case)
    d = lambda gs: [api.to_device(x) for x in gs]
    mu, data, cov, err = d(case.mu), d(case.data), d(case.cov), d([case.err_corr])[0]
    ctx.posterior_unit(mu, data, cov, err, precision)
    lay = G.Layout(case.nxp, case.nyp, case.nzp, 1)
    cs = api.Context(G.shard_case(case, nzp=lay.z(0)[1] - lay.z(0)[0]))
    cc = api.Context(G.shard_case(case, nyp=lay.y(0)[1] - lay.y(0)[0]))
    mu2, data2, cov2, err2 = d(case.mu), d(case.data), d(case.cov), d([case.err_corr])[0]
    G.posterior_unit_split(G.device_ops(cs, cc, precision, case.nzp), lay, 0, None, mu2, data2, cov2, err2)
    nx = case.nxp
    for a, b in zip(mu + data + cov, mu2 + data2 + cov2):
        assert torch.equal(a[..., :nx], b[..., :nx])


def test_loglik_over_split_grid_one_rank():
    """The split forward half and the per-shard functional give the one-GPU
    log marginal likelihood and gradients exactly."""
    case = synth.make_case(32, 24, 64, (0.0, 10.0, 20.0, 30.0, 40.0), 0.1, seed=14)
    ctx = api.Context(case, precision=api.FP64)
    d = lambda gs: [api.to_device(x) for x in gs]
    mu, data, cov, err = d(case.mu), d(case.data), d(case.cov), d([case.err_corr])[0]
    for g in mu:
        ctx.fft_r2c(g, api.PARAMETER)
    for g in data:
        ctx.fft_r2c(g, api.DATA)
    for g in cov + [err]:
        ctx.fft_r2c(g, api.COVARIANCE)
    L, gs, gv, gw, nf = ctx.loglik_grad(mu, data, cov, err)
    lay = G.Layout(case.nxp, case.nyp, case.nzp, 1)
    cs = api.Context(G.shard_case(case, nzp=case.nzp))
    cc = api.Context(G.shard_case(case, nyp=case.nyp), precision=api.FP64)
    ops = G.device_ops(cs, cc, api.FP64, case.nzp)
    m2, d2, c2, e2 = d(case.mu), d(case.data), d(case.cov), d([case.err_corr])[0]
    cols = G.spectra_to_columns(ops, lay, 0, None, m2, d2, c2, e2)
    L2, gs2, gv2, gw2, nf2 = G.loglik_grad_split(cc.loglik_grad, None, *cols)
    assert L2 == L and nf2 == nf
    assert np.array_equal(gs2, gs) and np.array_equal(gv2, gv) and np.array_equal(gw2, gw)
