"""Pins the CPU oracle (plain-C restatement) against the reference's own
numerics: the committed golden fixtures (made by tests/golden/make_golden.py
from oracle/_ref) and, when it is built, oracle/_ref itself."""
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests import golden_cases as GC


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


@pytest.mark.parametrize("name", GC.NAMES)
def test_solve_bitexact_vs_golden(name):
    """With the reference's spectra and kz tables, the restated FP32 solve
    reproduces the reference's lib_matr results bit for bit."""
    case, z = GC.load(name)
    mu, res, cov, fail = O.posterior_fp32_tables(case, GC.spectra(z), GC.tables(z), "orc")
    for a, b in zip(mu + res + cov, list(z["post_mu"]) + list(z["post_res"]) + list(z["post_cov"])):
        assert np.array_equal(bits(a), bits(b))
    assert fail == int(z["post_fail"])


@pytest.mark.parametrize("name", GC.NAMES)
def test_fft_vs_golden(name):
    """The restated 3-D R2C equals FFTW 2.1.2's to float rounding."""
    case, z = GC.load(name)
    n = (case.nxp, case.nyp, case.nzp)
    for g, ref, t in [(case.data[0], z["spec_data"][0], 1), (case.cov[1], z["spec_cov"][1], 3),
                      (case.mu[0], z["spec_mu"][0], 2)]:
        a = O.complex_view(O.fft_r2c(g, *n, t, "orc"), case.nxp)
        b = O.complex_view(ref, case.nxp)
        assert rel(a, b) < 5e-7


@pytest.mark.parametrize("name", GC.NAMES)
def test_tables_vs_golden(name):
    case, z = GC.load(name)
    wd, e1, e2, e3, inv = O.kz_tables(case, "orc")
    assert np.array_equal(inv, z["tab_inv"])
    assert np.array_equal(e3, z["tab_e3"])
    for a, b in [(wd, z["tab_wd"]), (e1, z["tab_e1"]), (e2, z["tab_e2"])]:
        assert np.abs(a - b).max() <= 2e-6 * max(np.abs(b).max(), 1e-30)


@pytest.mark.parametrize("name", GC.NAMES)
def test_unit_vs_golden(name):
    """The whole unit (restated FFT + solve) against the reference unit."""
    case, z = GC.load(name)
    mu, res, cov, fail = O.unit_fp32(case, "orc")
    nx = case.nxp
    for a, b in zip(mu + res + cov, list(z["unit_mu"]) + list(z["unit_res"]) + list(z["unit_cov"])):
        assert rel(a[..., :nx], b[..., :nx]) < 2e-5
    assert fail == int(z["unit_fail"])


def test_rng_bitexact_vs_golden():
    z = np.load(GC.HERE + "/rng_23665.npz")
    normals, state = O.rng_normal(23665, len(z["normals"]), "orc")
    assert np.array_equal(normals, z["normals"])
    assert state == int(z["state"])


@pytest.mark.parametrize("name", GC.NAMES)
def test_noise_and_filter_vs_golden(name):
    case, z = GC.load(name)
    nx, ny, nzp = case.nxp, case.nyp, case.nzp
    c = case.cnxp
    for s in range(3):
        g, _ = O.noise_fill(nx, ny, nzp, 1000 + s, "orc")
        assert np.array_equal(bits(g[..., :2 * c]), bits(z["sim_noise"][s][..., :2 * c]))
    sim, fail = O.sim_filter(nx, ny, nzp, list(z["post_cov"]), list(z["sim_noise"]), "orc")
    for a, b in zip(sim, z["sim"]):
        assert np.array_equal(bits(a[..., :2 * c]), bits(b[..., :2 * c]))
    assert fail == int(z["sim_fail"])


@pytest.mark.skipif(not O.have_ref(), reason="oracle/_ref not built (needs the reference tree)")
@pytest.mark.parametrize("shape,angles", [((16, 12, 32), (10.0, 20.0, 30.0)),
                                          ((20, 18, 30), (0.0, 10.0, 20.0, 30.0, 40.0))])
def test_solve_bitexact_vs_ref_live(shape, angles):
    from crava_b200 import synth
    case = synth.make_case(*shape, angles, 0.1, seed=3)
    sp = O.forward_spectra(case, "ref")
    tb = O.kz_tables(case, "ref")
    a = O.posterior_fp32_tables(case, sp, tb, "orc")
    b = O.posterior_fp32_tables(case, sp, tb, "ref")
    for x, y in zip(a[0] + a[1] + a[2], b[0] + b[1] + b[2]):
        assert np.array_equal(bits(x), bits(y))
    assert a[3] == b[3]


def test_fp64_twin_close_to_fp32():
    case, z = GC.load("c3_12x10x16")
    mu, res, cov, fail = O.posterior_fp64(case, GC.spectra(z))
    nx = case.nxp
    for a, b in zip(mu + cov, list(z["post_mu"]) + list(z["post_cov"])):
        assert rel(O.complex_view(b, nx), a) < 1e-4


def test_synt_seismic_vs_golden():
    """The restated synthetic seismic (double 1-D DFTs) equals the
    reference's trace loop with FFTW 2.1.2 to float rounding, with and
    without the padding taper and untouched traces."""
    z = np.load(os.path.join(GC.HERE, "synt_seismic.npz"))
    for name in ("c3_12x10x16", "c2_9x8x20_odd", "c5_10x8x24"):
        case, _ = GC.load(name)
        m = list(z[f"{name}_m"])
        k = 0
        while f"{name}_{k}_size" in z:
            nx, ny, nz = (int(v) for v in z[f"{name}_{k}_size"])
            out = O.synt_seismic(case, m, nx, ny, nz, "orc")
            for a, b in zip(out, z[f"{name}_{k}_out"]):
                assert rel(a, b) < 1e-6, (name, k)
            k += 1


def _corr_t(nzp, dt=4.0, t_range=20.0):
    i = np.arange(nzp // 2 + 2)
    return np.exp(-3.0 * (dt * i / t_range) ** 2).astype(np.float32)


@pytest.mark.parametrize("nzp,low_int_cut", [(32, 0), (128, 2), (300, 6), (512, 10)])
def test_circ_corr_t_restatement_and_library(nzp, low_int_cut):
    """computeCircCorrT + makeCircCorrTPosDef: the restatement and the
    library's host routine agree with each other and, when it is built,
    with the reference's FFTW version to float rounding."""
    from crava_b200 import api

    ct = _corr_t(nzp)
    a = O.circ_corr_t(ct, low_int_cut, nzp, "orc")
    b = api.circ_corr_t(ct, low_int_cut, nzp)
    assert np.abs(a - b).max() <= 2e-7
    if O.have_ref():
        r = O.circ_corr_t(ct, low_int_cut, nzp, "ref")
        assert np.abs(a - r).max() <= 1e-6


def test_prior_fills_match_synthetic_cases():
    """fillInParamCorr x var0 and fillInErrCorr restated equal the grids
    the seeded cases carry (same float operations) on every real cell."""
    from crava_b200 import synth

    for shape in [(16, 12, 32), (15, 16, 20)]:
        nx, ny, nz = shape
        case = synth.make_case(nx, ny, nz, (10.0,), 0.1, seed=1)
        cxy = synth.corr_xy(nx, ny, 25.0, 25.0, 500.0)
        circ = synth.circ_corr_t(nz, 4.0, 20.0, 5.0)
        cov = O.fill_prior_cov(nx, ny, nz, cxy, circ, 0.0, 0.0, case.var0)
        for g, h in zip(cov, case.cov):
            assert np.array_equal(bits(g[..., :nx]), bits(h[..., :nx]))
        assert np.array_equal(bits(O.fill_err_corr(nx, ny, nz, cxy, 0.0, 0.0)), bits(case.err_corr))


@pytest.mark.parametrize("shape", [(16, 12, 64), (15, 16, 20), (8, 8, 128)])
def test_nonconstant_thickness_tables_vs_ref(shape):
    """Tables of the non-constant-thickness branch (src/crava.cpp:1059-1083):
    restatement vs the reference's FFTW; the robust inverse wavelet modulus
    on the inverted planes (elsewhere it inverts spectrum values at the
    level of rounding noise and the solve does not read it)."""
    if not O.have_ref():
        pytest.skip("oracle/_ref not built")
    from crava_b200 import synth

    case = synth.make_case(*shape, (0.0, 15.0, 30.0), 0.1, seed=3)
    case.thickness_mode = 1
    case.min_rel_thick = 0.8
    a = O.kz_tables(case, "orc")
    b = O.kz_tables(case, "ref")
    assert np.array_equal(a[4], b[4])
    for x, y in zip(a[:3], b[:3]):
        assert np.abs(x - y).max() <= 1e-6 * np.abs(y).max()
    inv = b[4].astype(bool)
    assert np.abs(a[3][inv] - b[3][inv]).max() <= 1e-6 * np.abs(b[3][inv]).max()


# ---------------------------------------------------------------- State4D
def _golden_state4d():
    from tests import state4d_cases as SC
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "state4d.npz"))
    state = {k: [np.ascontiguousarray(g) for g in z[f"in_{k}"]] for k in SC.KEYS}
    return SC, z, state, list(z["mu_post"]), list(z["cov_post"])


def test_state4d_merge_split_bitexact_vs_golden():
    """merge / mergeCov and split restated reproduce the reference's
    lib_matr sequence (src/state4d.cpp:90-525) bit for bit, shortcut bins
    included."""
    SC, z, state, mu, cov = _golden_state4d()
    mmu = [np.zeros_like(mu[0]) for _ in range(3)]
    mcov = [np.zeros_like(mu[0]) for _ in range(6)]
    O.state4d_merge(state, mmu, mcov, "orc")
    for a, b in zip(mmu + mcov, list(z["merge_mu"]) + list(z["merge_cov"])):
        assert np.array_equal(bits(a), bits(b))
    st = SC.copy_state(state)
    fails = O.state4d_split(st, mu, cov, "orc")
    assert fails == int(z["split_fail"]) > 0
    for k in SC.KEYS:
        for a, b in zip(st[k], z[f"split_{k}"]):
            assert np.array_equal(bits(a), bits(b)), k


@pytest.mark.skipif(not O.have_ref(), reason="oracle/_ref not built (needs the reference tree)")
def test_state4d_vs_ref_live():
    from tests import state4d_cases as SC
    state, mu, cov = SC.random_state(20, 12, 16, seed=5, fail_every=41)
    out = {}
    for which in ("orc", "ref"):
        mmu = [np.zeros_like(mu[0]) for _ in range(3)]
        mcov = [np.zeros_like(mu[0]) for _ in range(6)]
        O.state4d_merge(state, mmu, mcov, which)
        st = SC.copy_state(state)
        f = O.state4d_split(st, mu, cov, which)
        out[which] = (mcov, st, f)
    assert out["orc"][2] == out["ref"][2] > 0
    for a, b in zip(out["orc"][0], out["ref"][0]):
        assert np.array_equal(bits(a), bits(b))
    for k in SC.KEYS:
        for a, b in zip(out["orc"][1][k], out["ref"][1][k]):
            assert np.array_equal(bits(a), bits(b))


def test_state4d_split_then_merge_gives_the_posterior():
    """After split, the merged current prior equals the inverted state it
    was split from, to float rounding: T B^H = I for T = [I I] and
    B = Sigma_cur^-1 T Sigma_full.  For the covariance this needs a
    Hermitian current covariance, which the reference's unconjugated
    lower-triangle copy keeps only when that covariance is real."""
    from tests import state4d_cases as SC
    state, mu, cov = SC.random_state(12, 8, 10, seed=9, fail_every=0, real_post_cov=True)
    st = SC.copy_state(state)
    assert O.state4d_split(st, mu, cov, "orc") == 0
    mmu = [np.zeros_like(mu[0]) for _ in range(3)]
    mcov = [np.zeros_like(mu[0]) for _ in range(6)]
    O.state4d_merge(st, mmu, mcov, "orc")
    for a, b in zip(mmu + mcov, mu + cov):
        assert rel(SC.to_complex(a), SC.to_complex(b)) < 1e-4


def test_state4d_evolve_restatement_vs_numpy():
    """evolve (src/state4d.cpp:527-730) against an independent float64
    numpy statement of E S E^T + C Re(lambda) and E mu + c s."""
    from tests import state4d_cases as SC
    nxp, nyp, nzp = 8, 6, 10
    state, _, _ = SC.random_state(nxp, nyp, nzp, seed=3)
    E, cm, cc = SC.evolution(4)
    lam = np.random.default_rng(5).standard_normal(SC.grid_shape(nxp, nyp, nzp)).astype(np.float32)
    scale = np.float32(np.sqrt(float(nxp * nyp * nzp)))
    st = SC.copy_state(state)
    O.state4d_evolve(st, E, cm, cc, lam, scale)
    c = SC.to_complex
    m = np.stack([c(g) for g in state["ms"] + state["md"]], -1).astype(np.complex128)
    n = m.shape[0]
    Sr, Si = np.zeros((n, 6, 6)), np.zeros((n, 6, 6))
    for r in range(6):
        for off, key in ((0, "ss"), (3, "dd")):
            v = c(state[key][r])
            p, q = SC.P[r] + off, SC.Q[r] + off
            Sr[:, p, q] = Sr[:, q, p] = v.real
            Si[:, p, q] = Si[:, q, p] = v.imag
    for l in range(3):
        for k in range(3):
            v = c(state["sd"][3 * l + k])
            Sr[:, l, k + 3] = Sr[:, k + 3, l] = v.real
            Si[:, l, k + 3] = Si[:, k + 3, l] = v.imag
    lr = c(lam).real.astype(np.float64)
    Nr = E @ Sr @ E.T + cc[None] * lr[:, None, None]
    Ni = E @ Si @ E.T
    mr = m.real @ E.T
    mr[0] += cm * float(scale)
    mi = m.imag @ E.T
    got = np.stack([c(g) for g in st["ms"] + st["md"]], -1)
    assert np.allclose(got.real, mr, rtol=1e-6, atol=1e-6) and np.allclose(got.imag, mi, rtol=1e-6, atol=1e-6)
    for r in range(6):
        for off, key in ((0, "ss"), (3, "dd")):
            v = c(st[key][r])
            p, q = SC.P[r] + off, SC.Q[r] + off
            assert np.allclose(v.real, Nr[:, p, q], rtol=1e-6, atol=1e-5)
            assert np.allclose(v.imag, Ni[:, p, q], rtol=1e-6, atol=1e-5)


def test_gen_exp_corr_restatement_vs_numpy():
    """fillInGenExpCorr (src/fftgrid.cpp:1167-1210) against numpy."""
    nxp, nyp, nzp, rx, ry, rz, gi, gj = 12, 10, 16, 4.0, 10.0 / 3.0, 5.0, 0.3, -0.2
    g = O.fill_gen_exp_corr(nxp, nyp, nzp, rx, ry, rz, gi, gj)
    i = np.arange(nxp)
    ci = np.where(i < nxp - i, i, i - nxp)
    j = np.arange(nyp)
    cj = np.where(j < nyp - j, j, j - nyp)
    k = np.arange(nzp)
    sub = (k[:, None, None] + ci[None, None, :] * np.float32(gi) + cj[None, :, None] * np.float32(gj))
    sub = (sub + nzp / 2.0) % nzp - nzp / 2.0
    ref = np.exp(-3.0 * np.sqrt((ci ** 2)[None, None, :] / rx ** 2 + (cj ** 2)[None, :, None] / ry ** 2
                                + sub ** 2 / rz ** 2))
    assert np.abs(g[..., :nxp] - ref).max() < 1e-6
    assert np.all(g[..., nxp:] == -99999.0)


# ------------------------------------------------ data / scale wavelet
def _divide_case(name):
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "divide.npz"))
    case, _ = GC.load(name)
    nx, ny, nz = (int(v) for v in z[f"{name}_size"])
    case.nz = nz
    shift = z[f"{name}_shift"] if f"{name}_shift" in z else None
    gain = z[f"{name}_gain"] if f"{name}_gain" in z else None
    return case, z, nx, ny, z[f"{name}_rel_thick"], float(z[f"{name}_dz"]), shift, gain


@pytest.mark.parametrize("name", ["c3_12x10x16", "c2_9x8x20_odd"])
def test_divide_data_vs_golden(name):
    """divideDataByScaleWavelet restated (double DFTs for FFTW, no drift of
    the global wavelet) against the reference's FFTW sequence: < 1e-5."""
    case, z, nx, ny, rt, dz, shift, gain = _divide_case(name)
    col = case.cov[0][:, 0, 0].copy()
    out = O.divide_data(case, case.data, col, rt, nx, ny, dz, shift, gain, "orc")
    for a, b, d in zip(out, z[f"{name}_out"], case.data):
        assert rel(a[..., :case.nxp], b[..., :case.nxp]) < 1e-5
        assert rel(b[..., :case.nxp], d[..., :case.nxp]) > 0.1  # the division did something


@pytest.mark.skipif(not O.have_ref(), reason="oracle/_ref not built (needs the reference tree)")
@pytest.mark.parametrize("name,local", [("c3_12x10x16", False), ("c2_9x8x20_odd", True)])
def test_multiply_data_vs_ref_live(name, local):
    """multiplyDataByScaleWaveletAndWriteToFile restated vs the reference's
    FFTW per-trace sequence: < 1e-5."""
    case, _ = GC.load(name)
    nx, ny = case.nxp - 2, case.nyp - 2
    rng = np.random.default_rng(12)
    rt = rng.uniform(0.7, 1.3, (case.nyp, case.nxp))
    shift = rng.uniform(-5, 5, (case.ntheta, ny, nx)).astype(np.float32) if local else None
    gain = rng.uniform(0.7, 1.3, (case.ntheta, ny, nx)).astype(np.float32) if local else None
    dz = float(np.float32(case.lz / case.nz))
    a = O.multiply_data(case, case.data, rt, nx, ny, dz, shift, gain, "orc")
    b = O.multiply_data(case, case.data, rt, nx, ny, dz, shift, gain, "ref")
    for x, y, d in zip(a, b, case.data):
        assert rel(x[:, :ny, :nx], y[:, :ny, :nx]) < 1e-5
        assert np.array_equal(x[:, ny:, :], d[:, ny:, :])
        assert rel(x[:, :ny, :nx], d[:, :ny, :nx]) > 0.1


def _interpolate_py(g, nxp, nyp, nzp, nx, ny, nz, thr):
    """FFTGrid::interpolateSeismic / interpolateTrace / extrapolateSeismic
    (src/fftgrid.cpp:2564-2731) restated again in Python with float32
    arithmetic, independently of the C restatement."""
    f32 = np.float32
    g = g.copy()
    at = lambda i, j: g[:, j, i]  # a trace, all nzp samples
    energy = np.zeros(nx * ny, f32)
    total = f32(0)
    for j in range(ny):
        for i in range(nx):
            e = f32(0)
            for k in range(nz):
                v = g[k, j, i]
                e = f32(e + f32(v * v))
            energy[i + nx * j] = e
            total = f32(total + e)
    limit = f32(f32(f32(thr) * total) / f32(nx * ny))
    flags = [0] * (nx * ny)
    flag, imin, imax, jmin, jmax, bad = 0, nx, 0, ny, 0, 0
    for j in range(ny):
        for i in range(nx):
            idx = i + nx * j
            cur = 1 if energy[idx] <= limit else 0
            bad += cur
            flags[idx] = flag + cur
            if cur:
                flag = 2
            else:
                imin, imax, jmin, jmax = min(imin, i), max(imax, i), min(jmin, j), max(jmax, j)

    def trace(idx, i, j):
        left = i > 0 and flags[idx - 1] % 2 == 0
        right = i < nx - 1 and flags[idx + 1] % 2 == 0
        up = j > 0 and flags[idx - nx] % 2 == 0
        down = j < ny - 1 and flags[idx + nx] % 2 == 0
        nt = left + right + up + down
        if nt > 1:
            m = at(i - 1, j).copy() if left else np.zeros(nzp, f32)
            for ok, (a, b) in ((right, (i + 1, j)), (up, (i, j - 1)), (down, (i, j + 1))):
                if ok:
                    m = (m + at(a, b)).astype(f32)
            g[:, j, i] = (m / f32(nt)).astype(f32)
            flags[idx] -= 1
        return flags[idx]

    cur = 0
    for j in range(ny):
        for i in range(nx):
            if flags[cur] % 2 == 1 and trace(cur, i, j) % 2 == 0:
                idx = cur - 1
                while idx >= 0 and flags[idx] > 1:
                    if flags[idx] % 2 == 1:
                        trace(idx, idx % nx, idx // nx)
                    idx -= 1
                idx = max(idx, 0) + 1
                while idx <= cur and flags[idx - 1] == 0:
                    if flags[idx] > 1:
                        flags[idx] -= 2
                    idx += 1
            cur += 1

    def fill(i, n, npad):
        if i < n:
            return i
        below, above = npad - i - 1, i - n + 1
        return max(n - above, n // 2) if above < below else min(below, n // 2)

    def dist(i, n, npad):
        if i < n:
            return f32(0)
        taper = f32(min(n, npad - n) / 2.1)
        below, above = npad - i, i - (n - 1)
        return f32(f32(above) / taper) if above < below else f32(f32(below) / taper)

    if imin <= imax:
        for j in range(nyp):
            rj = min(max(fill(j, ny, nyp), jmin), jmax)
            for i in range(nxp):
                if i < imin or i > imax or j < jmin or j > jmax:
                    ri = min(max(fill(i, nx, nxp), imin), imax)
                    for k in range(nzp):
                        dx, dy, dzz = dist(i, nx, nxp), dist(j, ny, nyp), dist(k, nz, nzp)
                        b = 1.0 - float(f32(dx * dx)) - float(f32(dy * dy)) - float(f32(dzz * dzz))
                        mult = f32(max(b, 0.0) ** 3)
                        g[k, j, i] = f32(mult * g[k, rj, ri])
    return g, bad


@pytest.mark.parametrize("bad", [[(3, 4), (4, 4), (5, 4), (0, 0), (11, 9), (5, 0), (6, 6), (7, 7), (6, 7)],
                                 [(0, j) for j in range(10)] + [(9, 9), (8, 8), (8, 9)]])
def test_interpolate_seismic_two_restatements(bad):
    """The C restatement of interpolateSeismic equals an independent Python
    one: the simbox traces bit for bit, the extrapolated padding to 1 ulp
    (pow of the two C libraries' callers)."""
    nxp, nyp, nzp, nx, ny, nz = 16, 12, 12, 12, 10, 9
    rng = np.random.default_rng(2)
    g = rng.standard_normal((nzp, nyp, 2 * (nxp // 2 + 1))).astype(np.float32)
    for n, (i, j) in enumerate(bad):
        g[:, j, i] = 0.0 if n % 2 == 0 else 1e-3
    a, ni, _ = O.interpolate_seismic(g, nxp, nyp, nzp, nx, ny, nz, 0.05)
    b, nb = _interpolate_py(g, nxp, nyp, nzp, nx, ny, nz, 0.05)
    assert ni == nb == len(bad)
    assert np.array_equal(a[:, :ny, :nx], b[:, :ny, :nx])
    d = np.abs(a.view(np.int32).astype(np.int64) - b.view(np.int32).astype(np.int64))
    assert d[..., :nxp].max() <= 1


@pytest.mark.skipif(not O.have_ref(), reason="oracle/_ref (the reference's FFTW build) is not built")
def test_synt_seismic_local_harness_vs_golden_and_constant_case():
    """The local-wavelet trace loop (stretch, shift, gain) on the reference's
    FFTW equals its golden fixture bit for bit, and with unit relative
    thickness and no shift or gain it equals the constant-thickness loop
    (itself pinned against synt_seismic.npz) bit for bit."""
    z = np.load(os.path.join(GC.HERE, "synt_local.npz"))
    for name in ("c3_12x10x16", "c2_9x8x20_odd"):
        case, _ = GC.load(name)
        nx, ny, nz = (int(v) for v in z[f"{name}_size"])
        m = list(z[f"{name}_m"])
        sh = z[f"{name}_shift"] if f"{name}_shift" in z else None
        ga = z[f"{name}_gain"] if f"{name}_gain" in z else None
        out = O.synt_seismic_local(case, m, z[f"{name}_rel_thick"], float(z[f"{name}_dz"]), sh, ga, nx, ny, nz)
        assert np.array_equal(np.stack(out), z[f"{name}_out"])
        ones = np.ones((case.nyp, case.nxp))
        a = O.synt_seismic_local(case, m, ones, float(z[f"{name}_dz"]), None, None, nx, ny, nz)
        b = O.synt_seismic(case, m, nx, ny, nz, "ref")
        assert all(np.array_equal(x, y) for x, y in zip(a, b))
