"""Seeded synthetic inversion cases in the reference's grid layout.

No public dataset is involved: every case is generated from a seed with the
formulas the reference uses to build its prior, noise model, wavelets and
reflection matrix, so the CPU oracle and the GPU path read identical bytes.

Recipe (reference file:line of each formula):
  * Prior variance Sigma0 from standard deviations and correlations
    (SeismicParametersHolder::setCorrelationParameters,
    src/seismicparametersholder.cpp:91-149).
  * Temporal correlation: Gaussian, corrT[i] = exp(-3 (i dt / range)^2) for
    i = 0 .. nzp/2+1 (src/modelgeneral.cpp:3858-3876 with power 2), made
    circular and positive definite with the low-frequency cut
    lowIntCut = floor(lowCut nzp 0.001 dt)
    (src/seismicparametersholder.cpp:430-499, src/modelgeneral.cpp:3961).
  * Lateral correlation: GenExpVario(pot=1, range, range) evaluated on the
    padded lateral grid (src/modelgeneral.cpp:4072-4110, src/vario.cpp:87-93).
  * The six prior covariance grids: circCorrT(k) * corrXY(i,j) * Sigma0_pq
    (FFTGrid::fillInParamCorr, src/fftgrid.cpp:1118-1164, with
    corrGradI = corrGradJ = 0; SeismicParametersHolder::initializeCorrelations
    :196-221).
  * Noise correlation grid: corrXY(i,j) on the k = 0 plane, zero elsewhere
    (FFTGrid::fillInErrCorr, src/fftgrid.cpp:1064-1116).
  * Truth: mu + a prior realisation (circulant filtering of white noise).
  * Wavelet: Ricker (src/wavelet.cpp:1354-1358) of 81 samples centred at t=0,
    stored in FFT order on nzp samples, with an optional per-angle scale.
  * Reflection matrix: PP Aki-Richards (src/modelavodynamic.cpp:875-911).
  * Seismic: conj(W) * D * sum_p A_lp m_p per trace (Crava::computeSyntSeismic,
    src/crava.cpp:1666-1719, no taper because unpadded = padded) plus white
    noise at a given fraction of the signal energy.
  * Noise variance per angle: dataVariance / S/N with S/N = (1+f)/f, and
    errThetaCov_lm = sqrt(ev_l ev_m) * exp(-3 |theta_l - theta_m| / 10 deg)
    (Crava::computeDataVariance / setupErrorCorrelation, src/crava.cpp:321-401).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

RMISSING = -99999.0
DATA, PARAMETER, COVARIANCE = 1, 2, 3


@dataclass
class Case:
    """One inversion case: parameters plus real-space padded grids."""

    nxp: int
    nyp: int
    nzp: int
    angles_deg: list
    dt: float
    low_cut: float
    high_cut: float
    wnc: float
    nz: int
    lz: float
    min_rel_thick: float
    wavelet: np.ndarray        # [ntheta, nzp] float32, FFT order
    A: np.ndarray              # [ntheta, 3] float32
    theta_cov: np.ndarray      # [ntheta, ntheta] float64
    var0: np.ndarray           # [3, 3] float64
    mu: list                   # 3 x float32 [nzp, nyp, rnxp]
    data: list                 # ntheta x float32 [nzp, nyp, rnxp]
    cov: list                  # 6 x float32 [nzp, nyp, rnxp]
    err_corr: np.ndarray       # float32 [nzp, nyp, rnxp]
    truth: list = field(default_factory=list)
    thickness_mode: int = 0    # 0 constant thickness, 1 non-constant (data divided by the wavelet)

    @property
    def ntheta(self):
        return len(self.angles_deg)

    @property
    def cnxp(self):
        return self.nxp // 2 + 1

    @property
    def rnxp(self):
        return 2 * self.cnxp

    def grids(self):
        """The 10+ntheta input grids in ABI order: mu(3), data, cov(6), err."""
        return list(self.mu) + list(self.data) + list(self.cov) + [self.err_corr]

    def copy(self):
        c = Case(**{k: getattr(self, k) for k in self.__dataclass_fields__})
        c.mu = [g.copy() for g in self.mu]
        c.data = [g.copy() for g in self.data]
        c.cov = [g.copy() for g in self.cov]
        c.err_corr = self.err_corr.copy()
        return c


def prior_var0(stds=(0.08, 0.12, 0.05), corr_ab=0.7, corr_ar=0.5, corr_br=0.4):
    s = np.array(stds, dtype=np.float64)
    c = np.array([[1.0, corr_ab, corr_ar], [corr_ab, 1.0, corr_br], [corr_ar, corr_br, 1.0]])
    v = (s[:, None] * s[None, :] * c).astype(np.float32)  # paramCov is float**
    return v.astype(np.float64)


def circ_corr_t(nzp, dt, t_range, low_cut):
    """computeCircCorrT + makeCircCorrTPosDef (seismicparametersholder.cpp:430-499)."""
    ncorr = nzp // 2 + 1 if nzp % 2 == 0 else nzp // 2
    i = np.arange(ncorr + 1, dtype=np.float64)
    corr_t = np.exp(-3.0 * (dt * i / t_range) ** 2).astype(np.float32)
    circ = np.zeros(nzp, dtype=np.float32)
    for k in range(nzp):
        refk = k if k < nzp // 2 + 1 else nzp - k
        circ[k] = corr_t[refk] if refk < len(corr_t) else 0.0
    low_int_cut = int(math.floor(low_cut * (nzp * 0.001 * dt)))
    spec = np.fft.rfft(circ.astype(np.float64))
    mag = np.abs(spec)
    mag[: low_int_cut + 1] = 0.0
    back = np.fft.irfft(mag, n=nzp) * nzp  # unnormalised inverse
    if back[0] <= 1e-5:
        raise ValueError("circular temporal correlation undefined")
    return (back / back[0]).astype(np.float32)


def corr_xy(nxp, nyp, dx, dy, lateral_range, power=1.0):
    """findCorrXYGrid with GenExpVario (modelgeneral.cpp:4072-4110)."""
    i = np.arange(nxp)
    j = np.arange(nyp)
    ri = np.where(i < nxp // 2 + 1, i, i - nxp).astype(np.float32) * np.float32(dx)
    rj = np.where(j < nyp // 2 + 1, j, j - nyp).astype(np.float32) * np.float32(dy)
    inv_r2 = np.float32(1.0 / (lateral_range * lateral_range))
    d2 = inv_r2 * ri[None, :] ** 2 + inv_r2 * rj[:, None] ** 2
    dist = np.sqrt(d2.astype(np.float32))
    return np.exp(-3.0 * np.power(dist.astype(np.float64), power)).astype(np.float32)  # [nyp, nxp]


def ricker(t_ms, peak_hz):
    """Wavelet::Ricker (src/wavelet.cpp:1354-1358)."""
    c = math.pi * math.pi * peak_hz * peak_hz * t_ms * t_ms * 1e-6
    return (1.0 - 2.0 * c) * math.exp(-c)


def ricker_fft_order(nzp, dt, peak_hz=25.0, nsamples=81, scale=1.0):
    w = np.zeros(nzp, dtype=np.float32)
    half = min(nsamples // 2, (nzp - 1) // 2)
    for n in range(-half, half + 1):
        w[n % nzp] = np.float32(ricker(n * dt, peak_hz)) * np.float32(scale)
    return w


def aki_richards_pp(angles_deg, vsvp=0.5):
    """setupDefaultReflectionMatrix, PP rows (modelavodynamic.cpp:895-900)."""
    A = np.zeros((len(angles_deg), 3), dtype=np.float32)
    v2 = vsvp * vsvp
    for l, a in enumerate(angles_deg):
        th = math.radians(a)
        s2 = math.sin(th) ** 2
        t2 = math.tan(th) ** 2
        A[l] = [(1.0 + t2) / 2.0, -4 * v2 * s2, (1.0 - 4.0 * v2 * s2) / 2.0]
    return A


def _padded(real_xyz, nxp, fill=RMISSING):
    """[nzp, nyp, nxp] -> padded [nzp, nyp, 2*(nxp//2+1)] float32."""
    nzp, nyp, _ = real_xyz.shape
    rnxp = 2 * (nxp // 2 + 1)
    out = np.full((nzp, nyp, rnxp), fill, dtype=np.float32)
    out[:, :, :nxp] = real_xyz
    return out


def make_case(nxp=64, nyp=64, nzp=128, angles_deg=(10.0, 20.0, 30.0), noise_frac=0.10,
              seed=1, wavelet_scale_range=None, dx=25.0, dy=25.0, dt=4.0,
              t_range=20.0, lateral_range=500.0, low_cut=5.0, high_cut=55.0,
              wnc=0.1, peak_hz=25.0, vsvp=0.5, angular_range_deg=10.0,
              mu_const=(math.log(3000.0), math.log(1500.0), math.log(2.3)),
              keep_truth=False):
    """Builds one seeded case; unpadded = padded (nx = nxp, nz = nzp)."""
    rng = np.random.default_rng(seed)
    nt = len(angles_deg)
    var0 = prior_var0()
    circ = circ_corr_t(nzp, dt, t_range, low_cut)
    cxy = corr_xy(nxp, nyp, dx, dy, lateral_range)
    base = (circ[:, None, None] * cxy[None, :, :]).astype(np.float32)  # [nzp, nyp, nxp]
    pairs = [(0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2)]
    cov = [_padded(base * np.float32(var0[p, q]), nxp) for p, q in pairs]
    err = np.zeros((nzp, nyp, nxp), dtype=np.float32)
    err[0] = cxy
    err_corr = _padded(err, nxp)

    # truth = mu + prior realisation
    lam = np.abs(np.fft.rfftn(base.astype(np.float64), axes=(0, 1, 2)).real)
    filt = np.sqrt(lam)
    L0 = np.linalg.cholesky(var0)
    fields = []
    for _ in range(3):
        w = rng.standard_normal((nzp, nyp, nxp))
        fields.append(np.fft.irfftn(filt * np.fft.rfftn(w), s=(nzp, nyp, nxp), axes=(0, 1, 2)))
    truth = []
    for p in range(3):
        f = sum(L0[p, q] * fields[q] for q in range(3))
        truth.append(mu_const[p] + f)

    A = aki_richards_pp(angles_deg, vsvp)
    scales = np.ones(nt)
    if wavelet_scale_range is not None:
        lo, hi = wavelet_scale_range
        scales = lo + (hi - lo) * rng.random(nt)
    wav = np.stack([ricker_fft_order(nzp, dt, peak_hz, 81, s) for s in scales]).astype(np.float32)

    kz = np.arange(nzp // 2 + 1)
    dop = -1.0 + np.exp(2j * np.pi * kz / nzp)  # FFT of [-1,0,..,0,1]
    data = []
    data_var = np.zeros(nt)
    for l in range(nt):
        imp = sum(float(A[l, p]) * truth[p] for p in range(3))
        W = np.fft.rfft(wav[l].astype(np.float64))
        spec = np.fft.rfft(imp, axis=0) * (np.conj(W) * dop)[:, None, None]
        sig = np.fft.irfft(spec, n=nzp, axis=0)
        sig_var = float(np.mean(sig * sig))
        noisy = sig + rng.standard_normal(sig.shape) * math.sqrt(noise_frac * sig_var)
        noisy = noisy.astype(np.float32)
        nzv = noisy[noisy != 0.0].astype(np.float64)
        data_var[l] = float(np.float32(np.sum(nzv * nzv) / max(nzv.size, 1)))
        data.append(_padded(noisy, nxp, fill=0.0))

    sn = (1.0 + noise_frac) / noise_frac
    ev = (data_var / sn).astype(np.float32)
    th = np.radians(np.asarray(angles_deg, dtype=np.float64)).astype(np.float32)
    rng_ang = math.radians(angular_range_deg)
    theta_cov = np.zeros((nt, nt))
    for a in range(nt):
        for b in range(nt):
            dth = float(np.float32(th[a] - th[b]))
            c = float(np.float32(math.exp(-3.0 * abs(dth) / rng_ang)))
            theta_cov[a, b] = float(np.float32(math.sqrt(ev[a]) * math.sqrt(ev[b]) * c))

    mu = [_padded(np.full((nzp, nyp, nxp), mu_const[p], dtype=np.float32), nxp) for p in range(3)]
    case = Case(nxp=nxp, nyp=nyp, nzp=nzp, angles_deg=list(angles_deg), dt=dt,
                low_cut=low_cut, high_cut=high_cut, wnc=wnc, nz=nzp, lz=nzp * dt,
                min_rel_thick=1.0, wavelet=wav, A=A, theta_cov=theta_cov, var0=var0,
                mu=mu, data=data, cov=cov, err_corr=err_corr)
    if keep_truth:
        case.truth = [t.astype(np.float32) for t in truth]
    return case


def config_small(seed=1, noise_frac=0.10):
    """64x64x128, 3 angles at 10/20/30 degrees."""
    return make_case(64, 64, 128, (10.0, 20.0, 30.0), noise_frac, seed)


def config_full(seed=2, noise_frac=0.10):
    """256x256x512, 5 angles at 0..40 degrees, wavelet scale U[0.8, 1.2]."""
    return make_case(256, 256, 512, (0.0, 10.0, 20.0, 30.0, 40.0), noise_frac, seed,
                     wavelet_scale_range=(0.8, 1.2))
