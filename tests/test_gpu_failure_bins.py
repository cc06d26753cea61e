"""Planted failures in the per-bin solve.

The reference keeps the prior at a bin whose data covariance M does not
factor (src/crava.cpp:1109-1111): lib_matrCholCpx fails when M00 <= 0 or
when a diagonal entry or pivot of M / M00 is <= 1e-20
(libs/lib/lib_matr.c:20, 103-105, 114, 145), and its comparisons let a NaN
through, so a NaN in a bin's inputs gives NaN outputs rather than a
failure.  This file plants, on the host, into the spectra of a small case:

* bins whose prior S is indefinite so that M00 <= 0 (zero diagonal, large
  off-diagonals whose products with the reflectivity row are negative, and
  a zero noise spectrum);
* bins whose M00 > 0 but a later pivot is negative (large S00 and S12);
* NaN bins: a NaN data spectrum and a NaN noise spectrum at inverted bins,
  a NaN covariance spectrum at a band-gated bin.

Every form must report the oracle's failed-bin count, keep the prior
exactly at the failed bins (mean and data untouched, covariance = the
prior of that form's arithmetic), and produce non-finite outputs exactly
where the oracle does, with nonfinite_bins counting those bins.
"""
import numpy as np
import pytest

from crava_b200 import api, synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu

PAIRS = [(0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2)]


def _noise_cov(case, tables, k, lam):
    wd, e1, e2, e3, inv = tables
    wnc = np.float64(np.float32(case.wnc))
    th = case.theta_cov
    a, b, c = (t[k].astype(np.complex128) for t in (e1, e2, e3))
    N = 0.5 * (1.0 - wnc) * th * lam * (np.outer(a, a.conj()) + np.outer(b, b.conj()))
    return N + np.diag(np.diag(th) * wnc * c.real ** 2)


def _M(case, tables, k, S, lam):
    K = tables[0][k].astype(np.complex128)[:, None] * case.A.astype(np.float64)
    return K @ S @ K.conj().T + _noise_cov(case, tables, k, lam)


def _fail_kind(M):
    """lib_matrCholCpx's failure rule in double: 'm00', 'pivot' or None."""
    f = M[0, 0].real
    if f <= 0:
        return "m00"
    A = M / f
    n = len(A)
    L = np.zeros_like(A)
    for i in range(n):
        if A[i, i].real <= 1e-20:
            return "pivot"
        for j in range(i):
            L[i, j] = (A[i, j] - np.sum(L[i, :j] * L[j, :j].conj())) / L[j, j]
        d = A[i, i].real - np.sum(np.abs(L[i, :i]) ** 2)
        if d <= 1e-20:
            return "pivot"
        L[i, i] = np.sqrt(d)
    return None


def _plant():
    case = synth.make_case(24, 20, 64, (10.0, 20.0, 30.0, 40.0), 0.1, seed=61)
    sp = O.forward_spectra(case, "orc")
    tables = O.kz_tables(case, "orc")
    inv = tables[4]
    cv = lambda g: O.complex_view(g, case.nxp)
    band = [k for k in range(case.nzp) if inv[k]]
    gated = [k for k in range(case.nzp) if not inv[k]]
    big = 10.0 * max(np.abs(cv(g)).max() for g in sp["cov"])
    plants = {"m00": [], "pivot": [], "nan": []}
    rng = np.random.default_rng(7)
    used = set()

    def pick(planes):
        while True:
            b = (int(rng.choice(planes)), int(rng.integers(case.nyp)), int(rng.integers(case.cnxp)))
            if b not in used:
                used.add(b)
                return b

    # M00 <= 0: S_pp = 0, S01 = S12 = x, S02 = 0, no noise spectrum
    for _ in range(6):
        k, j, i = pick(band)
        x = big
        for t, v in enumerate([0.0, 0.0, 0.0, x, 0.0, x]):
            cv(sp["cov"][t])[k, j, i] = v
        cv(sp["err"])[k, j, i] = 0.0
        S = np.array([[0, x, 0], [x, 0, x], [0, x, 0]], complex)
        assert _fail_kind(_M(case, tables, k, S, 0.0)) == "m00"
        plants["m00"].append((k, j, i))
    # M00 > 0, a later pivot negative: S00 = S12 = x, the rest 0
    for _ in range(6):
        k, j, i = pick(band)
        x = big
        for t, v in enumerate([x, 0.0, 0.0, 0.0, 0.0, x]):
            cv(sp["cov"][t])[k, j, i] = v
        lam = abs(float(cv(sp["err"])[k, j, i].real))
        S = np.array([[x, 0, 0], [0, 0, x], [0, x, 0]], complex)
        assert _fail_kind(_M(case, tables, k, S, lam)) == "pivot"
        plants["pivot"].append((k, j, i))
    # NaN: data at an inverted bin, noise at an inverted bin, covariance at a gated bin
    k, j, i = pick(band)
    cv(sp["data"][1])[k, j, i] = complex(np.nan, 0.0)
    plants["nan"].append((k, j, i))
    k, j, i = pick(band)
    cv(sp["err"])[k, j, i] = complex(np.nan, 0.0)
    plants["nan"].append((k, j, i))
    k, j, i = pick(gated)
    cv(sp["cov"][2])[k, j, i] = complex(np.nan, 0.0)
    plants["nan"].append((k, j, i))
    return case, sp, tables, plants


@pytest.fixture(scope="module")
def planted():
    return _plant()


def _run(case, sp, tables, prec):
    ctx = api.Context(case)
    ctx.set_kz_tables(tables)
    d = lambda gs: [api.to_device(g) for g in gs]
    mu, data, cov, err = d(sp["mu"]), d(sp["data"]), d(sp["cov"]), d([sp["err"]])[0]
    ctx.posterior(mu, data, cov, err, prec)
    st = ctx.stats()
    cvt = lambda gs: [api.complex_view(g.cpu().numpy(), case.nxp) for g in gs]
    return cvt(mu), cvt(data), cvt(cov), st


def _nonfinite_bins(outs):
    bad = np.zeros(outs[0].shape, bool)
    for o in outs:
        bad |= ~np.isfinite(o)
    return bad


@pytest.mark.parametrize("prec", [api.FP64, api.MIXED])
def test_failed_bins_keep_the_prior(planted, prec):
    case, sp, tables, plants = planted
    omu, ores, ocov, ofail = O.posterior_fp64(case, sp)
    assert ofail == len(plants["m00"]) + len(plants["pivot"])
    mu, res, cov, st = _run(case, sp, tables, prec)
    assert st.chol_fail_bins == ofail
    cv = lambda g: O.complex_view(g, case.nxp)
    # the prior of this form's arithmetic at a failed bin
    if prec == api.FP64:
        prior = [o.astype(np.complex64) for o in ocov]  # |Re c / S0| S0 in double, rounded
    else:
        prior = O.posterior_fp32(case, sp, "orc")[2]  # the reference's float operations
        prior = [cv(g) for g in prior]
    for b in plants["m00"] + plants["pivot"]:
        for q in range(3):
            assert mu[q][b] == cv(sp["mu"][q])[b]
        for l in range(case.ntheta):
            assert res[l][b] == cv(sp["data"][l])[b]
        for t in range(6):
            assert cov[t][b] == prior[t][b], (b, t)
    # non-finite outputs exactly where the oracle has them
    gpu_bad = _nonfinite_bins(mu + res + cov)
    ora_bad = _nonfinite_bins(omu + ores + ocov)
    assert np.array_equal(gpu_bad, ora_bad)
    assert st.nonfinite_bins == int(ora_bad.sum()) == len(plants["nan"])
    for b in plants["nan"]:
        assert ora_bad[b]


def test_failed_bins_fp32_form_equals_reference_order(planted):
    """The FP32 form with the plants equals the reference-order restatement
    bit for bit, NaNs included."""
    case, sp, tables, plants = planted
    omu, ores, ocov, ofail = O.posterior_fp32(case, sp, "orc")
    mu, res, cov, st = _run(case, sp, tables, api.FP32)
    assert st.chol_fail_bins == ofail == len(plants["m00"]) + len(plants["pivot"])
    cv = lambda g: O.complex_view(g, case.nxp)
    for a, b in zip(mu + res + cov, omu + ores + ocov):
        assert np.array_equal(a, cv(b), equal_nan=True)
