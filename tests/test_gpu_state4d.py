"""The time-lapse state (State4D, src/state4d.cpp) on the device: merge and
split bit for bit against the reference's lib_matr sequence (the committed
fixture and the restatement), evolve against the float64 restatement, the
generalised exponential correlation, and advanceTime as a whole."""
import os

import numpy as np
import pytest
import torch

from crava_b200 import api, synth
from oracle import oracle as O
from tests import state4d_cases as SC

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def _ctx(nxp, nyp, nzp):
    return api.Context(synth.make_case(nxp, nyp, nzp, (10.0, 20.0), 0.1, seed=2))


def _dev_state(state):
    return {k: [api.to_device(g) for g in state[k]] for k in SC.KEYS}


def _host_state(dstate):
    return {k: [g.cpu().numpy() for g in dstate[k]] for k in SC.KEYS}


def test_merge_and_split_vs_reference_fixture():
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "state4d.npz"))
    nxp, nyp, nzp = (int(v) for v in z["shape"])
    ctx = _ctx(nxp, nyp, nzp)
    state = {k: [np.ascontiguousarray(g) for g in z[f"in_{k}"]] for k in SC.KEYS}
    mu = [api.to_device(g) for g in z["mu_post"]]
    cov = [api.to_device(g) for g in z["cov_post"]]
    ds = _dev_state(state)
    mmu = [torch.zeros_like(mu[0]) for _ in range(3)]
    mcov = [torch.zeros_like(mu[0]) for _ in range(6)]
    ctx.state4d_merge(ds, mmu, mcov)
    for a, b in zip(mmu + mcov, list(z["merge_mu"]) + list(z["merge_cov"])):
        assert np.array_equal(bits(a.cpu().numpy()), bits(b))
    fails = ctx.state4d_split(ds, mu, cov)
    assert fails == int(z["split_fail"]) > 0
    assert ctx.stats().chol_fail_bins == fails
    got = _host_state(ds)
    for k in SC.KEYS:
        for a, b in zip(got[k], z[f"split_{k}"]):
            assert np.array_equal(bits(a), bits(b)), k


@pytest.mark.parametrize("shape", [(64, 48, 96), (15, 1, 20)])
def test_merge_split_evolve_vs_restatement(shape):
    nxp, nyp, nzp = shape
    ctx = _ctx(nxp, nyp, nzp)
    state, mu, cov = SC.random_state(nxp, nyp, nzp, seed=17, fail_every=101)
    ds = _dev_state(state)
    # mergeCov alone (mu NULL) and merge
    mcov = [torch.zeros(SC.grid_shape(nxp, nyp, nzp), device="cuda") for _ in range(6)]
    ctx.state4d_merge(ds, None, mcov)
    omu = [np.zeros_like(mu[0]) for _ in range(3)]
    ocov = [np.zeros_like(mu[0]) for _ in range(6)]
    O.state4d_merge(state, omu, ocov, "orc")
    for a, b in zip(mcov, ocov):
        assert np.array_equal(bits(a.cpu().numpy()), bits(b))
    # split
    dmu, dcov = [api.to_device(g) for g in mu], [api.to_device(g) for g in cov]
    f = ctx.state4d_split(ds, dmu, dcov)
    of = O.state4d_split(state, mu, cov, "orc")
    assert f == of > 0
    got = _host_state(ds)
    for k in SC.KEYS:
        for a, b in zip(got[k], state[k]):
            assert np.array_equal(bits(a), bits(b)), k
    # evolve: float64 products in the same order, no contraction
    E, cm, cc = SC.evolution(6)
    lam = np.random.default_rng(7).standard_normal(SC.grid_shape(nxp, nyp, nzp)).astype(np.float32)
    ctx.state4d_evolve(ds, E, cm, cc, api.to_device(lam))
    O.state4d_evolve(state, E, cm, cc, lam, np.float32(np.sqrt(float(nxp * nyp * nzp))))
    got = _host_state(ds)
    for k in SC.KEYS:
        for a, b in zip(got[k], state[k]):
            assert np.array_equal(bits(a), bits(b)), k


def test_gen_exp_corr_vs_restatement():
    nxp, nyp, nzp = 40, 30, 64
    ctx = _ctx(nxp, nyp, nzp)
    g = torch.zeros(SC.grid_shape(nxp, nyp, nzp), device="cuda")
    for rx, ry, rz, gi, gj in [(40 / 3.0, 10.0, 50.0, 0.0, 0.0), (5.0, 7.5, 5.0, 0.25, -0.4)]:
        ctx.fill_gen_exp_corr(rx, ry, rz, gi, gj, g)
        ref = O.fill_gen_exp_corr(nxp, nyp, nzp, rx, ry, rz, gi, gj)
        got = g.cpu().numpy()
        # exp() of CUDA and of the C library may differ in the last bit of
        # a double; after rounding to float the grids agree to 1 ulp
        d = np.abs(bits(got).astype(np.int64) - bits(ref).astype(np.int64))
        assert d.max() <= 1
    with pytest.raises(api.CravaGpuError):
        ctx.fill_gen_exp_corr(0.0, 1.0, 1.0, 0.0, 0.0, g)


def _physical_state(nxp, nyp, nzp, seed):
    """A state whose spectra are transforms of real grids (Hermitian across
    bins, as a real state's are): covariances c(x) S0_pq of one symmetric
    correlation grid c and a fixed 6x6 S0, random real means; the inverted
    current state is 0.6 times the merged prior covariance and random
    real-field means."""
    rng = np.random.default_rng(seed)
    G = rng.standard_normal((6, 6))
    S0 = G @ G.T / 6.0 + 0.5 * np.eye(6)
    c = O.fill_gen_exp_corr(nxp, nyp, nzp, nxp / 4.0, nyp / 4.0, 6.0, 0.0, 0.0)
    lam = SC.to_complex(O.fft_r2c(c, nxp, nyp, nzp, api.COVARIANCE, "orc"))
    shape = SC.grid_shape(nxp, nyp, nzp)
    g = lambda v: np.ascontiguousarray(v.astype(np.complex64)).view(np.float32).reshape(shape).copy()

    def field(kind):
        x = rng.standard_normal(shape).astype(np.float32)
        return O.fft_r2c(x, nxp, nyp, nzp, kind, "orc")

    state = {"ms": [field(api.PARAMETER) for _ in range(3)], "md": [field(api.PARAMETER) for _ in range(3)],
             "ss": [g(lam * S0[SC.P[r], SC.Q[r]]) for r in range(6)],
             "dd": [g(lam * S0[SC.P[r] + 3, SC.Q[r] + 3]) for r in range(6)],
             "sd": [g(lam * S0[l, k + 3]) for l in range(3) for k in range(3)]}
    C = S0[:3, :3] + S0[3:, 3:] + S0[3:, :3] + S0[:3, 3:]
    mu = [field(api.PARAMETER) for _ in range(3)]
    cov = [None] * 6
    for r in range(6):
        cov[SC.UNIT[r]] = g(0.6 * lam * C[SC.P[r], SC.Q[r]])
    return state, mu, cov


def test_advance_time_vs_restatement():
    """advanceTime (src/modelgeneral.cpp:4722-4736): split, evolve with the
    transformed time-increment correlation, merge, inverse transforms; two
    steps (vertical range 50, then 5)."""
    nxp, nyp, nzp, nx, ny = 24, 20, 32, 20, 16
    ctx = _ctx(nxp, nyp, nzp)
    state, mu, cov = _physical_state(nxp, nyp, nzp, seed=23)
    E, cm, cc = SC.evolution(8)
    ds = _dev_state(state)
    dmu, dcov = [api.to_device(g) for g in mu], [api.to_device(g) for g in cov]
    work = torch.zeros(SC.grid_shape(nxp, nyp, nzp), device="cuda")
    for step in (0, 1):
        hmu = [g.cpu().numpy() for g in dmu]
        hcov = [g.cpu().numpy() for g in dcov]
        state = _host_state(ds)
        f = ctx.advance_time(ds, step, nx, ny, E, cm, cc, dmu, dcov, work)
        # the same steps through the restatement, from the same inputs
        of = O.state4d_split(state, hmu, hcov, "orc")
        assert f == of
        lam = O.fill_gen_exp_corr(nxp, nyp, nzp, float(np.float32(nx)) / 3.0, float(np.float32(ny)) / 3.0,
                                  50.0 if step == 0 else 5.0, 0.0, 0.0)
        lam = O.fft_r2c(lam, nxp, nyp, nzp, api.COVARIANCE, "orc")
        O.state4d_evolve(state, E, cm, cc, lam, np.float32(np.sqrt(float(nxp * nyp * nzp))))
        omu = [np.zeros_like(mu[0]) for _ in range(3)]
        ocov = [np.zeros_like(mu[0]) for _ in range(6)]
        O.state4d_merge(state, omu, ocov, "orc")
        got = _host_state(ds)
        for k in SC.KEYS:
            for a, b in zip(got[k], state[k]):
                assert rel(SC.to_complex(a), SC.to_complex(b)) < 1e-5, (step, k)
        tmu = [O.fft_c2r(g.copy(), nxp, nyp, nzp, api.PARAMETER, "orc") for g in omu]
        tcov = [O.fft_c2r(g.copy(), nxp, nyp, nzp, api.COVARIANCE, "orc") for g in ocov]
        for a, b in zip(dmu + dcov, tmu + tcov):
            assert rel(a.cpu().numpy()[..., :nxp], b[..., :nxp]) < 1e-5, step
        # the next step starts from the merged prior, back in the Fourier domain
        for g in dmu:
            ctx.fft_r2c(g, api.PARAMETER)
        for g in dcov:
            ctx.fft_r2c(g, api.COVARIANCE)


def test_state4d_rejects_bad_arguments():
    ctx = _ctx(16, 12, 32)
    state, mu, cov = SC.random_state(16, 12, 32, seed=1)
    ds = _dev_state(state)
    dmu, dcov = [api.to_device(g) for g in mu], [api.to_device(g) for g in cov]
    E, cm, cc = SC.evolution(1)
    work = torch.zeros_like(dmu[0])
    with pytest.raises(api.CravaGpuError):
        ctx.advance_time(ds, -1, 16, 12, E, cm, cc, dmu, dcov, work)  # negative time step
    with pytest.raises(api.CravaGpuError):
        ctx.advance_time(ds, 0, 17, 12, E, cm, cc, dmu, dcov, work)  # nx above nxp
    with pytest.raises(api.CravaGpuError):
        ctx.fill_gen_exp_corr(4.0, 4.0, 4.0, float("inf"), 0.0, work)
