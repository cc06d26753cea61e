"""Posterior realisations on the GPU: the per-bin Cholesky filter against
the reference's own arithmetic (golden fixtures), the Hermitian rules and
the distribution of the seeded noise, and the statistics of realisations
against the posterior covariance they are drawn from."""
import numpy as np
import pytest
import torch

from crava_b200 import api, synth
from tests import golden_cases as GC

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


@pytest.mark.parametrize("name", GC.NAMES)
def test_filter_bitexact_vs_reference(name):
    """Same noise in, same posterior spectra in: the GPU filter equals the
    reference's lib_matrCholCpx + lib_matrProdCholVec bit for bit."""
    case, z = GC.load(name)
    ctx = api.Context(case)
    cov = [api.to_device(g) for g in z["post_cov"]]
    seeds = [api.to_device(g) for g in z["sim_noise"]]
    ctx.sim_filter(cov, seeds)
    st = ctx.stats()
    c = case.cnxp
    for g, ref in zip(seeds, z["sim"]):
        assert np.array_equal(bits(g.cpu().numpy()[..., :2 * c]), bits(ref[..., :2 * c]))
    assert st.chol_fail_bins == int(z["sim_fail"])


@pytest.mark.parametrize("shape", [(16, 12, 32), (15, 10, 21), (64, 48, 96), (16, 1, 64)])
def test_noise_hermitian_rules(shape):
    nx, ny, nz = shape
    case = synth.make_case(nx, ny, nz, (10.0,), 0.1, seed=1)
    ctx = api.Context(case)
    g = torch.zeros((nz, ny, 2 * (nx // 2 + 1)), dtype=torch.float32, device="cuda")
    ctx.noise_fill(g, 1234, 7)
    c = api.complex_view(g.cpu().numpy(), nx).reshape(-1)
    cnxp = nx // 2 + 1
    for i in range(c.size):
        xs = i % cnxp
        if xs == 0 or (xs == cnxp - 1 and i % 2 == 1):
            jk = i // cnxp
            j, k = jk % ny, jk // ny
            jc = 0 if j == 0 else ny - j
            kc = 0 if k == 0 else nz - k
            jkc = jc + kc * ny
            if jkc == jk:
                assert c[i].imag == 0.0
            elif jkc < jk:
                assert c[i] == np.conj(c[jkc * cnxp + xs])
    # regular bins: both parts N(0, 1/2)
    reg = np.array([c[i] for i in range(c.size) if 0 < i % cnxp < cnxp - 1])
    for part in (reg.real, reg.imag):
        assert abs(part.mean()) < 5 * np.sqrt(0.5 / part.size)
        assert abs(part.var() - 0.5) < 6 * 0.5 * np.sqrt(2.0 / part.size)


def test_noise_is_reproducible_and_streams_differ():
    case = synth.make_case(16, 12, 32, (10.0,), 0.1, seed=1)
    ctx = api.Context(case)
    shape = (32, 12, 18)
    a = torch.zeros(shape, device="cuda"); b = torch.zeros(shape, device="cuda")
    c = torch.zeros(shape, device="cuda")
    ctx.noise_fill(a, 99, 3); ctx.noise_fill(b, 99, 3); ctx.noise_fill(c, 99, 4)
    assert torch.equal(a, b) and not torch.equal(a, c)


def test_realisations_match_posterior_covariance():
    """Spectra of (realisation - posterior mean) have covariance S_post."""
    case = synth.make_case(32, 24, 64, (10.0, 20.0, 30.0), 0.1, seed=5)
    ctx = api.Context(case)
    d = lambda gs: [api.to_device(g) for g in gs]
    mu, data, cov, err = d(case.mu), d(case.data), d(case.cov), d([case.err_corr])[0]
    for g in data + mu:
        pass
    # transformed means/stacks as Crava::Crava leaves them, then the solve
    for g in mu:
        ctx.fft_r2c(g, api.PARAMETER)
    for g in data:
        ctx.fft_r2c(g, api.DATA)
    for g in cov + [err]:
        ctx.fft_r2c(g, api.COVARIANCE)
    ctx.posterior(mu, data, cov, err, api.FP64)
    for g in mu:
        ctx.fft_c2r(g, api.PARAMETER)
    R = 12
    outs = [torch.zeros_like(mu[0]) for _ in range(3 * R)]
    ctx.simulate(cov, mu, 2024, 0, outs)
    nx = case.nxp
    inner = slice(1, nx // 2)  # exclude the kx = 0 and Nyquist planes
    S = [api.complex_view(g.cpu().numpy(), nx)[..., inner].reshape(-1) for g in cov]
    P = np.zeros((S[0].size, 3, 3), complex)
    idx = {(0, 0): 0, (1, 1): 1, (2, 2): 2, (0, 1): 3, (0, 2): 4, (1, 2): 5}
    for (p, q), t in idx.items():
        P[:, p, q] = S[t]
        P[:, q, p] = np.conj(S[t])
    ev = np.linalg.eigvalsh(P)
    ok = ev[:, 0] > 1e-6 * ev[:, 2].clip(min=1e-30)   # well-conditioned bins only
    L = np.linalg.cholesky(P[ok])
    acc = np.zeros((3, 3), complex)
    n = 0
    for r in range(R):
        zs = []
        for p in range(3):
            t = outs[3 * r + p] - mu[p]
            ctx.fft_r2c(t, api.PARAMETER)
            zs.append(api.complex_view(t.cpu().numpy(), nx)[..., inner].reshape(-1))
        zv = np.stack(zs, axis=1)[ok][..., None]
        w = np.linalg.solve(L, zv)[..., 0]          # whitened: iid CN(0, I) expected
        acc += np.einsum("np,nq->pq", w, np.conj(w))
        n += w.shape[0]
    C = acc / n
    assert n > 10000
    for p in range(3):
        assert abs(C[p, p].real - 1.0) < 0.03, C
        for q in range(3):
            if p != q:
                assert abs(C[p, q]) < 0.03, C


def test_batched_realisations_equal_single_calls():
    """Realisation r of one call of 11 (batches of 8 + 3) equals the call
    that makes realisation r alone: each realisation depends only on (seed, r)."""
    case = synth.make_case(16, 12, 32, (10.0, 25.0), 0.1, seed=3)
    ctx = api.Context(case)
    d = lambda gs: [api.to_device(g) for g in gs]
    mu, cov = d(case.mu), d(case.cov)
    for g in cov:
        ctx.fft_r2c(g, api.COVARIANCE)
    R = 11
    outs = [torch.zeros_like(mu[0]) for _ in range(3 * R)]
    ctx.simulate(cov, mu, 77, 5, outs)
    for r in (0, 7, 8, 10):
        one = [torch.zeros_like(mu[0]) for _ in range(3)]
        ctx.simulate(cov, mu, 77, 5 + r, one)
        for p in range(3):
            assert torch.equal(one[p], outs[3 * r + p]), (r, p)
    assert not torch.equal(outs[0], outs[3])
