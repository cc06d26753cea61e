"""The Woodbury form of the per-bin posterior and the precision of its parts.

A float64 numpy statement of the form the FP64 solve uses
(crava_b200/csrc/woodbury.cuh: per plane N = Dg^1/2 V (lambda diag(m) + I)
V^H Dg^1/2, per bin P = sum_i c_i W_i^H W_i, S_post = Z^H Z with
Z = R^-1 LS^T, mu_post = mu + S_post W^H diag(c) T (d - K mu)) is checked
against the reference's matrix form (src/crava.cpp:1104-1130:
X = M^-1 K S, S_post = S - (K S)^H X, mu_post = mu + X^H (d - K mu),
M = K S K^H + N) on the oracle's spectra.  The same statement with chosen
steps rounded to float32 shows why a mixed FP32 + FP64-refinement variant
of the Woodbury form saves little: the data term must stay FP64 at high
SNR, and with it FP64 only the 3x3 chain can move to FP32.
Test infrastructure only (CPU, numpy)."""
import numpy as np

from crava_b200 import synth
from oracle import oracle as O

PAIRS = [(0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2)]
C64, C32 = np.complex128, np.complex64


def _inverted_bins(case):
    sp = O.forward_spectra(case, "orc")
    wd, e1, e2, e3, inv = O.kz_tables(case, "orc")
    cv = lambda g: O.complex_view(g, case.nxp).astype(C64)
    mu = np.stack([cv(g) for g in sp["mu"]], -1)
    d = np.stack([cv(g) for g in sp["data"]], -1)
    cov = np.stack([cv(g) for g in sp["cov"]], -1)
    err = cv(sp["err"])
    nt = case.ntheta
    th = case.theta_cov
    wnc = np.float64(np.float32(case.wnc))
    A = case.A.astype(np.float64)
    for k in np.nonzero(inv)[0]:
        e1k, e2k, e3k = e1[k].astype(C64), e2[k].astype(C64), e3[k].astype(np.float64)
        E = 0.5 * (1 - wnc) * th * (np.outer(e1k, e1k.conj()) + np.outer(e2k, e2k.conj()))
        Dg = wnc * np.diag(th) * e3k ** 2
        K = wd[k].astype(C64)[:, None] * A
        mk, dk = mu[k].reshape(-1, 3), d[k].reshape(-1, nt)
        ck, lam = cov[k].reshape(-1, 6), np.abs(err[k].reshape(-1).real)
        S = np.zeros((mk.shape[0], 3, 3))
        for t, (p, q) in enumerate(PAIRS):
            s0 = case.var0[p, q]
            S[:, p, q] = S[:, q, p] = np.abs(ck[:, t].real / s0) * s0
        yield mk, dk, S, lam, E, Dg, K


def _matrix_form(mk, dk, S, lam, E, Dg, K):
    M = np.einsum("lp,bpq,mq->blm", K, S, K.conj()) + lam[:, None, None] * E + np.diag(Dg)
    KS = np.einsum("lp,bpq->blq", K, S)
    X = np.linalg.solve(M, KS)
    r = dk - mk @ K.T
    mp = mk + np.einsum("blp,bl->bp", X.conj(), r)
    Sp = S - np.einsum("blp,blq->bpq", KS.conj(), X)
    return mp, dk - mp @ K.T, Sp


def _woodbury(mk, dk, S, lam, E, Dg, K, data32=False, chain32=False, refine=False):
    rs = 1.0 / np.sqrt(Dg)
    m, V = np.linalg.eigh(rs[:, None] * E * rs[None, :])
    T = V.conj().T * rs[None, :]
    W = T @ K
    c = 1.0 / (lam[:, None] * m[None, :] + 1.0)
    LS = np.linalg.cholesky(S)
    if data32:  # the data term and P in float32
        c32, T32, W32, K32 = c.astype(np.float32), T.astype(C32), W.astype(C32), K.astype(C32)
        r = (dk.astype(C32) - mk.astype(C32) @ K32.T).astype(C64)
        g = ((c32 * (r.astype(C32) @ T32.T)) @ W32.conj()).astype(C64)
        P = np.einsum("bi,ip,iq->bpq", c32.astype(C32), W32.conj(), W32).astype(C64)
    else:
        r = dk - mk @ K.T
        g = (c * (r @ T.T)) @ W.conj()
        P = np.einsum("bi,ip,iq->bpq", c.astype(C64), W.conj(), W)
    Q = np.einsum("bkp,bkq->bpq", LS.astype(C64), P @ LS.astype(C64))
    IQ = np.eye(3)[None] + Q
    ft = C32 if chain32 else C64
    R = np.linalg.cholesky(IQ.astype(ft))
    Rh = np.swapaxes(R.conj(), 1, 2)
    LSt = np.swapaxes(LS, 1, 2).astype(ft)
    Z = np.linalg.solve(R, LSt)
    Sp = np.einsum("bkp,bkq->bpq", Z.conj(), Z).astype(C64)
    b = np.einsum("bqp,bq->bp", LS.astype(C64), g)[..., None]
    y = np.linalg.solve(Rh, np.linalg.solve(R, b.astype(ft))).astype(C64)
    if refine:  # one FP64 refinement step of (I + Q) y = LS^T g
        e = b - IQ @ y
        y = y + np.linalg.solve(Rh, np.linalg.solve(R, e.astype(ft))).astype(C64)
    dm = (LS.astype(C64) @ y)[..., 0]
    mp = mk + dm
    return mp, r - dm @ K.T, Sp


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _collect(case, fn):
    outs = [fn(*bins) for bins in _inverted_bins(case)]
    return [np.concatenate([o[i].reshape(o[i].shape[0], -1) for o in outs]) for i in range(3)]


def test_woodbury_equals_matrix_form():
    case = synth.make_case(24, 20, 64, (0.0, 10.0, 20.0, 30.0, 40.0), 0.1, seed=41)
    ref = _collect(case, _matrix_form)
    got = _collect(case, _woodbury)
    for a, b in zip(got, ref):
        assert _rel(a, b) < 1e-9


def test_mixed_woodbury_needs_the_fp64_data_term():
    """At 1 % noise (high SNR) the float32 data term leaves mean errors
    orders of magnitude above those of the variant that keeps it in FP64
    and moves only the 3x3 chain to FP32 with one FP64 refinement of the
    mean; the latter's covariance error is the FP32 chain's."""
    case = synth.make_case(24, 20, 64, (0.0, 10.0, 20.0, 30.0, 40.0), 0.01, seed=42)
    ref = _collect(case, _woodbury)
    all32 = _collect(case, lambda *b: _woodbury(*b, data32=True, chain32=True))
    mix = _collect(case, lambda *b: _woodbury(*b, chain32=True, refine=True))
    e_all = [_rel(a, r) for a, r in zip(all32, ref)]
    e_mix = [_rel(a, r) for a, r in zip(mix, ref)]
    assert e_mix[0] < 1e-8 and e_mix[1] < 1e-8          # mean, residual: refined
    assert e_mix[2] < 1e-5                               # covariance: the FP32 chain
    assert e_all[0] > 100 * e_mix[0] and e_all[1] > 100 * e_mix[1]
