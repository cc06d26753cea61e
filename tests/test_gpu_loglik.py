"""Log marginal likelihood and its hand-written adjoint: the kernel's value
against an FP64 numpy restatement, its gradients against central finite
differences (step 1e-3 relative, FP64) of the same functional, and the
torch.autograd wrapper against the direct call."""
import numpy as np
import pytest
import torch

from crava_b200 import api, synth
from crava_b200.loglik import log_marginal

pytestmark = pytest.mark.gpu

ANGLES5 = (0.0, 10.0, 20.0, 30.0, 40.0)


def _spectra(ctx, case):
    d = lambda gs: [api.to_device(g) for g in gs]
    mu, data, cov, err = d(case.mu), d(case.data), d(case.cov), d([case.err_corr])[0]
    for g in mu:
        ctx.fft_r2c(g, api.PARAMETER)
    for g in data:
        ctx.fft_r2c(g, api.DATA)
    for g in cov + [err]:
        ctx.fft_r2c(g, api.COVARIANCE)
    return mu, data, cov, err


def _wavelet_spectrum(case):
    W = np.fft.fft(case.wavelet.astype(np.float64), axis=-1)  # [nt, nzp]
    return W[:, : case.nzp // 2 + 1].T.copy()                 # [cnzp, nt]


def loglik_numpy(ctx, case, grids, scale, noise, spec):
    """FP64 restatement of the functional (see crava_gpu_loglik_grad)."""
    nx, nzp, nt = case.nxp, case.nzp, case.ntheta
    cv = lambda t: api.complex_view(t.cpu().numpy(), nx).astype(np.complex128)
    mu = np.stack([cv(g) for g in grids[0]], -1)           # [z, y, x, 3]
    d = np.stack([cv(g) for g in grids[1]], -1)            # [z, y, x, nt]
    c6 = [cv(g).real for g in grids[2]]
    ec = cv(grids[3]).real
    _, e1, e2, e3, inv = ctx.kz_tables()
    e1, e2, e3 = e1.astype(np.complex128), e2.astype(np.complex128), e3.astype(np.float64)
    v0 = case.var0
    vv = [v0[0, 0], v0[1, 1], v0[2, 2], v0[0, 1], v0[0, 2], v0[1, 2]]
    r6 = [np.abs(c / v) * v if v != 0 else np.abs(c) for c, v in zip(c6, vv)]
    S = np.empty(c6[0].shape + (3, 3))
    for t, (p, q) in enumerate([(0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2)]):
        S[..., p, q] = r6[t]
        S[..., q, p] = r6[t]
    A = case.A.astype(np.float64)
    B = np.einsum("lp,...pq,mq->...lm", A, S, A)
    k = np.arange(nzp)
    D = np.exp(2j * np.pi * k / nzp) - 1.0
    cn = nzp // 2 + 1
    Wfull = np.empty((nzp, nt), np.complex128)
    Wfull[:cn] = spec
    Wfull[cn:] = np.conj(spec[1: nzp - cn + 1][::-1])
    w = scale[None, :] * D[:, None] * np.conj(Wfull)        # [nzp, nt]
    th = case.theta_cov * np.sqrt(np.outer(noise, noise) / np.outer(np.diag(case.theta_cov),
                                                                     np.diag(case.theta_cov)))
    cc = 0.5 * (1.0 - np.float64(np.float32(case.wnc))) * np.abs(ec)
    n12 = e1[:, :, None] * np.conj(e1[:, None, :]) + e2[:, :, None] * np.conj(e2[:, None, :])
    N = cc[..., None, None] * th * n12[:, None, None]
    wnc = np.float64(np.float32(case.wnc))
    N = N + np.einsum("l,zl,lm->zlm", np.diag(th) * wnc, e3 ** 2, np.eye(nt))[:, None, None]
    ww = w[:, :, None] * np.conj(w[:, None, :])
    M = ww[:, None, None] * B + N
    idx = np.arange(nt)
    M[..., idx, idx] = M[..., idx, idx].real
    r = d - w[:, None, None, :] * np.einsum("lq,...q->...l", A, mu)
    L = np.linalg.cholesky(M)
    logdet = 2.0 * np.log(np.real(np.diagonal(L, axis1=-2, axis2=-1))).sum(-1)
    al = np.linalg.solve(M, r[..., None])[..., 0]
    quad = np.real(np.sum(np.conj(r) * al, -1))
    kx = np.arange(case.cnxp)
    ck = np.where((kx == 0) | (2 * kx == nx), 1.0, 2.0)
    term = (-logdet - quad) * ck
    return float(term[inv.astype(bool)].sum())


@pytest.fixture(scope="module")
def small():
    case = synth.make_case(32, 24, 64, ANGLES5, 0.1, seed=12)
    ctx = api.Context(case, precision=api.FP64)
    grids = _spectra(ctx, case)
    return case, ctx, grids


def test_value_matches_fp64_restatement(small):
    case, ctx, grids = small
    nt = case.ntheta
    spec = _wavelet_spectrum(case)
    rng = np.random.default_rng(0)
    for scale, noise in [(np.ones(nt), np.diag(case.theta_cov).copy()),
                         (rng.uniform(0.8, 1.2, nt), np.diag(case.theta_cov) * rng.uniform(0.5, 2.0, nt))]:
        L, *_ = ctx.loglik_grad(*grids, scale, noise, spec)
        ref = loglik_numpy(ctx, case, grids, scale, noise, spec)
        assert abs(L - ref) <= 1e-10 * abs(ref), (L, ref)
    # defaults: scale 1, theta_cov diagonal, the context's own wavelets
    L0, *_ = ctx.loglik_grad(*grids)
    ref0 = loglik_numpy(ctx, case, grids, np.ones(nt), np.diag(case.theta_cov), spec)
    assert abs(L0 - ref0) <= 1e-9 * abs(ref0)


def _fd_check(f, x0, grad, idx, rel_step=1e-3, tol=1e-4, mag=None):
    """Central differences with step rel_step * |x0| (or rel_step * mag for
    components whose own value may be zero, e.g. the imaginary part of a
    real wavelet spectrum)."""
    for i in idx:
        h = rel_step * (abs(x0[i]) if mag is None else mag[i])
        xp, xm = x0.copy(), x0.copy()
        xp[i] += h
        xm[i] -= h
        fd = (f(xp) - f(xm)) / (2 * h)
        scale = max(abs(grad[i]), abs(fd), 1e-12)
        assert abs(fd - grad[i]) <= tol * scale, (i, fd, grad[i])


def test_gradients_match_finite_differences(small):
    case, ctx, grids = small
    nt = case.ntheta
    spec = _wavelet_spectrum(case)
    scale = np.array([0.9, 1.1, 1.0, 0.95, 1.05])
    noise = np.diag(case.theta_cov) * np.array([1.2, 0.8, 1.0, 1.5, 0.7])
    L, gs, gv, gw, nf = ctx.loglik_grad(*grids, scale, noise, spec)
    assert nf == 0
    _fd_check(lambda s: ctx.loglik_grad(*grids, s, noise, spec)[0], scale, gs, range(nt))
    _fd_check(lambda v: ctx.loglik_grad(*grids, scale, v, spec)[0], noise, gv, range(nt))
    # wavelet spectrum: real and imaginary parts of in-band bins
    _, _, _, _, inv = ctx.kz_tables()
    cn = case.nzp // 2 + 1
    band = [k for k in range(1, cn - 1) if inv[k]]
    picks = [(band[0], 0), (band[len(band) // 2], 2), (band[-1], 4), (band[len(band) // 3], 1)]
    flat = np.stack([spec.real, spec.imag], -1).reshape(-1)
    gflat = np.stack([gw.real, gw.imag], -1).reshape(-1)
    f = lambda x: ctx.loglik_grad(*grids, scale, noise, x.reshape(cn, nt, 2))[0]
    idx = [(k * nt + l) * 2 + part for k, l in picks for part in (0, 1)]
    mag = np.repeat(np.abs(spec).reshape(-1), 2)
    _fd_check(f, flat, gflat, idx, mag=mag)


def test_autograd_wrapper(small):
    case, ctx, grids = small
    nt = case.ntheta
    spec = _wavelet_spectrum(case)
    s = torch.ones(nt, dtype=torch.float64, requires_grad=True)
    v = torch.tensor(np.diag(case.theta_cov), requires_grad=True)
    w = torch.tensor(np.stack([spec.real, spec.imag], -1), requires_grad=True)
    L = log_marginal(ctx, grids, s, v, w)
    L.backward()
    L2, gs, gv, gw, _ = ctx.loglik_grad(*grids, s.detach().numpy(), v.detach().numpy(), spec)
    assert float(L.detach()) == L2
    assert np.array_equal(s.grad.numpy(), gs) and np.array_equal(v.grad.numpy(), gv)
    assert np.array_equal(w.grad.numpy(), np.stack([gw.real, gw.imag], -1))
