"""ctypes front end of the CPU oracle.  TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
import this module.  It loads

  * oracle/build/libcrava_oracle.so  -- the plain-C restatement (orc_*), and
  * oracle/_ref/libcrava_ref.so      -- the reference's own FFTW 2.1.2,
    lib_matr.c and random.cpp driven by ref_harness.cpp (ref_*), when built.

Arrays are numpy float32 grids in the padded layout [nzp, nyp, 2*(nxp/2+1)].
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORC_LIB = os.path.join(HERE, "build", "libcrava_oracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libcrava_ref.so")
# The reference source tree the harness is compiled from (build time only;
# nothing reads it at run time): CRAVA_REFERENCE_SRC, else its location in
# the build container.
REF_SRC = os.environ.get("CRAVA_REFERENCE_SRC", "/root/reference")

F32P = C.POINTER(C.c_float)
F64P = C.POINTER(C.c_double)


class Params(C.Structure):
    """Same layout as crava_gpu_params (include/crava_gpu.h)."""

    _fields_ = [
        ("nxp", C.c_int), ("nyp", C.c_int), ("nzp", C.c_int), ("ntheta", C.c_int),
        ("nz", C.c_int), ("precision", C.c_int),
        ("lz", C.c_double), ("min_rel_thick", C.c_double),
        ("low_cut", C.c_float), ("high_cut", C.c_float), ("wnc", C.c_float),
        ("thickness_mode", C.c_int),
        ("wavelet", F32P), ("wavelet_norm", F32P), ("A", F32P),
        ("theta_cov", F64P), ("var0", F64P),
    ]


def build(ref: bool | None = None) -> None:
    """Compiles the restatement, and the reference harness when the
    reference source tree is present (or ref=True)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    if ref is None:
        ref = os.path.isdir(REF_SRC)
    if ref:
        if not os.path.isfile(os.path.join(REF_SRC, "libs", "lib", "lib_matr.c")):
            raise FileNotFoundError(f"reference source tree not found at {REF_SRC} "
                                    "(set CRAVA_REFERENCE_SRC)")
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={REF_SRC}", "-j8"], check=True)


_libs = {}


def _load(which: str):
    if which in _libs:
        return _libs[which]
    path = ORC_LIB if which == "orc" else REF_LIB
    if which == "orc" and not os.path.exists(path):
        build(ref=False)
    if not os.path.exists(path):
        raise FileNotFoundError(path)
    lib = C.CDLL(path)
    p = which
    vp = C.c_void_p
    for name in ("fft_r2c", "fft_c2r"):
        f = getattr(lib, f"{p}_{name}")
        f.argtypes = [F32P, C.c_int, C.c_int, C.c_int, C.c_int]
        f.restype = C.c_int
    f = getattr(lib, f"{p}_kz_tables")
    f.argtypes = [C.POINTER(Params), F32P, F32P, F32P, F32P, C.POINTER(C.c_int)]
    f.restype = C.c_int
    for name in ("posterior_fp32", "unit_fp32"):
        f = getattr(lib, f"{p}_{name}")
        f.argtypes = [C.POINTER(Params), C.POINTER(F32P), C.POINTER(F32P), C.POINTER(F32P),
                      F32P, C.POINTER(C.c_longlong)]
        f.restype = C.c_int
    f = getattr(lib, f"{p}_posterior_fp32_t")
    f.argtypes = [C.POINTER(Params), F32P, F32P, F32P, F32P, C.POINTER(C.c_int),
                  C.POINTER(F32P), C.POINTER(F32P), C.POINTER(F32P), F32P, C.POINTER(C.c_longlong)]
    f.restype = C.c_int
    f = getattr(lib, f"{p}_rng_fill_normal")
    f.argtypes = [C.c_uint, F64P, C.c_longlong]
    f.restype = C.c_uint
    f = getattr(lib, f"{p}_noise_fill")
    f.argtypes = [F32P, C.c_int, C.c_int, C.c_int, C.c_uint]
    f.restype = C.c_uint
    f = getattr(lib, f"{p}_sim_filter")
    f.argtypes = [C.c_int, C.c_int, C.c_int, C.POINTER(F32P), C.POINTER(F32P), C.POINTER(C.c_longlong)]
    f.restype = C.c_int
    f = getattr(lib, f"{p}_circ_corr_t")
    f.argtypes = [F32P, C.c_int, C.c_int, C.c_int, F32P]
    f.restype = C.c_int
    if which == "orc":
        f = lib.orc_fill_prior_cov
        f.argtypes = [C.c_int, C.c_int, C.c_int, F32P, F32P, C.c_float, C.c_float, F64P, C.POINTER(F32P)]
        f.restype = C.c_int
        f = lib.orc_fill_err_corr
        f.argtypes = [C.c_int, C.c_int, C.c_int, F32P, C.c_float, C.c_float, F32P]
        f.restype = C.c_int
    f = getattr(lib, f"{p}_synt_seismic")
    f.argtypes = [C.c_int] * 7 + [F32P, F32P, C.POINTER(F32P), C.POINTER(F32P)]
    f.restype = C.c_int
    if which == "orc":
        f = lib.orc_posterior_fp64
        f.argtypes = [C.POINTER(Params), C.POINTER(F32P), C.POINTER(F32P), C.POINTER(F32P), F32P,
                      C.POINTER(F64P), C.POINTER(F64P), C.POINTER(F64P), C.POINTER(C.c_longlong)]
        f.restype = C.c_int
        f = lib.orc_sim_filter_fp64
        f.argtypes = [C.c_int, C.c_int, C.c_int, C.POINTER(F32P), C.POINTER(F32P), C.POINTER(C.c_longlong)]
        f.restype = C.c_int
    if which == "ref":
        f = lib.ref_synt_seismic_local
        f.argtypes = [C.c_int] * 7 + [F32P, F32P, C.POINTER(F32P), F64P, C.c_float, F32P, F32P,
                                      C.POINTER(F32P)]
        f.restype = C.c_int
    f = getattr(lib, f"{p}_divide_data")
    f.argtypes = [C.POINTER(Params), C.POINTER(F32P), F32P, F64P, C.c_int, C.c_int, C.c_float, F32P, F32P]
    f.restype = C.c_int
    f = getattr(lib, f"{p}_multiply_data")
    f.argtypes = [C.POINTER(Params), C.POINTER(F32P), F64P, C.c_int, C.c_int, C.c_float, F32P, F32P]
    f.restype = C.c_int
    if which == "orc":
        f = lib.orc_interpolate_seismic
        f.argtypes = [F32P] + [C.c_int] * 6 + [C.c_float, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        f.restype = C.c_int
    s4 = [C.POINTER(F32P)] * 7
    f = getattr(lib, f"{p}_state4d_merge")
    f.argtypes = [C.c_longlong] + s4
    f.restype = None
    f = getattr(lib, f"{p}_state4d_split")
    f.argtypes = [C.c_longlong] + s4
    f.restype = C.c_longlong
    if which == "orc":
        f = lib.orc_state4d_evolve
        f.argtypes = [C.c_longlong] + [C.POINTER(F32P)] * 5 + [F64P, F64P, F64P, F32P, C.c_float]
        f.restype = None
        f = lib.orc_fill_gen_exp_corr
        f.argtypes = [C.c_int] * 3 + [C.c_double] * 3 + [C.c_float, C.c_float, F32P]
        f.restype = C.c_int
    _libs[which] = lib
    return lib


def have_ref() -> bool:
    return os.path.exists(REF_LIB)


def _fp(a):
    assert a.dtype == np.float32 and a.flags.c_contiguous
    return a.ctypes.data_as(F32P)


def _dp(a):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(F64P)


def _ptrs(arrs, conv=_fp, typ=F32P):
    return (typ * len(arrs))(*[conv(a) for a in arrs])


def make_params(case, keep=None):
    """Params struct for a synth.Case; `keep` collects the owned arrays."""
    keep = [] if keep is None else keep
    wav = np.ascontiguousarray(case.wavelet, dtype=np.float32)
    A = np.ascontiguousarray(case.A, dtype=np.float32)
    th = np.ascontiguousarray(case.theta_cov, dtype=np.float64)
    v0 = np.ascontiguousarray(case.var0, dtype=np.float64)
    keep += [wav, A, th, v0]
    p = Params(case.nxp, case.nyp, case.nzp, case.ntheta, case.nz, 0, case.lz,
               case.min_rel_thick, case.low_cut, case.high_cut, case.wnc,
               int(getattr(case, "thickness_mode", 0)),
               _fp(wav), None, _fp(A), _dp(th), _dp(v0))
    return p, keep


def fft_r2c(grid, nxp, nyp, nzp, type_, which="orc"):
    g = np.ascontiguousarray(grid, dtype=np.float32).copy()
    getattr(_load(which), f"{which}_fft_r2c")(_fp(g), nxp, nyp, nzp, type_)
    return g


def fft_c2r(grid, nxp, nyp, nzp, type_, which="orc"):
    g = np.ascontiguousarray(grid, dtype=np.float32).copy()
    getattr(_load(which), f"{which}_fft_c2r")(_fp(g), nxp, nyp, nzp, type_)
    return g


def kz_tables(case, which="orc"):
    p, keep = make_params(case)
    n = case.nzp * case.ntheta
    wd = np.zeros(2 * n, np.float32); e1 = np.zeros(2 * n, np.float32)
    e2 = np.zeros(2 * n, np.float32); e3 = np.zeros(n, np.float32)
    inv = np.zeros(case.nzp, np.int32)
    rc = getattr(_load(which), f"{which}_kz_tables")(
        C.byref(p), _fp(wd), _fp(e1), _fp(e2), _fp(e3), inv.ctypes.data_as(C.POINTER(C.c_int)))
    assert rc == 0
    cpx = lambda a: a.view(np.complex64).reshape(case.nzp, case.ntheta)
    return cpx(wd), cpx(e1), cpx(e2), e3.reshape(case.nzp, case.ntheta), inv


def posterior_fp32(case, spectra, which="orc"):
    """Fourier-domain solve.  spectra: dict mu/data/cov/err of float32
    padded grids already transformed.  Returns (mu, data(res), cov, fails)."""
    p, keep = make_params(case)
    mu = [g.copy() for g in spectra["mu"]]
    data = [g.copy() for g in spectra["data"]]
    cov = [g.copy() for g in spectra["cov"]]
    err = np.ascontiguousarray(spectra["err"], dtype=np.float32)
    fails = C.c_longlong(0)
    rc = getattr(_load(which), f"{which}_posterior_fp32")(
        C.byref(p), _ptrs(mu), _ptrs(data), _ptrs(cov), _fp(err), C.byref(fails))
    assert rc == 0
    return mu, data, cov, fails.value


def posterior_fp32_tables(case, spectra, tables, which="orc"):
    """As posterior_fp32 but with given per-kz tables (wd, e1, e2, e3, inv)."""
    p, keep = make_params(case)
    wd, e1, e2, e3, inv = [np.ascontiguousarray(t) for t in tables]
    f32 = lambda a: np.ascontiguousarray(a.view(np.float32) if a.dtype == np.complex64 else a,
                                         dtype=np.float32)
    wd, e1, e2, e3 = f32(wd), f32(e1), f32(e2), f32(e3)
    inv = np.ascontiguousarray(inv, dtype=np.int32)
    mu = [g.copy() for g in spectra["mu"]]
    data = [g.copy() for g in spectra["data"]]
    cov = [g.copy() for g in spectra["cov"]]
    err = np.ascontiguousarray(spectra["err"], dtype=np.float32)
    fails = C.c_longlong(0)
    rc = getattr(_load(which), f"{which}_posterior_fp32_t")(
        C.byref(p), _fp(wd), _fp(e1), _fp(e2), _fp(e3), inv.ctypes.data_as(C.POINTER(C.c_int)),
        _ptrs(mu), _ptrs(data), _ptrs(cov), _fp(err), C.byref(fails))
    assert rc == 0
    return mu, data, cov, fails.value


def posterior_fp64(case, spectra):
    """FP64 twin.  Returns complex128 arrays [nzp, nyp, cnxp]."""
    p, keep = make_params(case)
    shape = (case.nzp, case.nyp, case.cnxp)
    mk = lambda n: [np.zeros(shape + (2,), np.float64) for _ in range(n)]
    mu_o, cov_o, res_o = mk(3), mk(6), mk(case.ntheta)
    fails = C.c_longlong(0)
    rc = _load("orc").orc_posterior_fp64(
        C.byref(p), _ptrs(spectra["mu"]), _ptrs(spectra["data"]), _ptrs(spectra["cov"]),
        _fp(np.ascontiguousarray(spectra["err"], dtype=np.float32)),
        _ptrs(mu_o, _dp, F64P), _ptrs(cov_o, _dp, F64P), _ptrs(res_o, _dp, F64P), C.byref(fails))
    assert rc == 0
    cv = lambda lst: [a.view(np.complex128)[..., 0] for a in lst]
    return cv(mu_o), cv(res_o), cv(cov_o), fails.value


def forward_spectra(case, which="orc"):
    """Forward transforms of every input grid with the reference scalings."""
    n = (case.nxp, case.nyp, case.nzp)
    return {
        "mu": [fft_r2c(g, *n, 2, which) for g in case.mu],
        "data": [fft_r2c(g, *n, 1, which) for g in case.data],
        "cov": [fft_r2c(g, *n, 3, which) for g in case.cov],
        "err": fft_r2c(case.err_corr, *n, 3, which),
    }


def unit_fp32(case, which="orc"):
    """The whole timed unit on real grids; returns (mu, res, cov, fails)."""
    p, keep = make_params(case)
    mu = [g.copy() for g in case.mu]
    data = [g.copy() for g in case.data]
    cov = [g.copy() for g in case.cov]
    err = case.err_corr.copy()
    fails = C.c_longlong(0)
    rc = getattr(_load(which), f"{which}_unit_fp32")(
        C.byref(p), _ptrs(mu), _ptrs(data), _ptrs(cov), _fp(err), C.byref(fails))
    assert rc == 0
    return mu, data, cov, fails.value


def rng_normal(seed, n, which="orc"):
    out = np.zeros(n, np.float64)
    s = getattr(_load(which), f"{which}_rng_fill_normal")(seed, _dp(out), n)
    return out, s


def noise_fill(nxp, nyp, nzp, seed, which="orc"):
    g = np.zeros((nzp, nyp, 2 * (nxp // 2 + 1)), np.float32)
    s = getattr(_load(which), f"{which}_noise_fill")(_fp(g), nxp, nyp, nzp, seed)
    return g, s


def sim_filter(nxp, nyp, nzp, cov, seeds, which="orc", fp64=False):
    sd = [s.copy() for s in seeds]
    fails = C.c_longlong(0)
    lib = _load(which)
    fn = lib.orc_sim_filter_fp64 if fp64 else getattr(lib, f"{which}_sim_filter")
    rc = fn(nxp, nyp, nzp, _ptrs(cov), _ptrs(sd), C.byref(fails))
    assert rc == 0
    return sd, fails.value


def synt_seismic(case, m, nx=None, ny=None, nz=None, which="orc"):
    """Synthetic seismic of the real padded grids m = (alpha, beta, rho):
    one real padded grid per angle (Crava::computeSyntSeismic)."""
    lib = _load(which)
    nx = case.nxp if nx is None else nx
    ny = case.nyp if ny is None else ny
    nz = case.nz if nz is None else nz
    mm = [np.ascontiguousarray(g, dtype=np.float32) for g in m]
    out = [np.zeros_like(mm[0]) for _ in range(case.ntheta)]
    A = np.ascontiguousarray(case.A, dtype=np.float32)
    wav = np.ascontiguousarray(case.wavelet, dtype=np.float32)
    rc = getattr(lib, f"{which}_synt_seismic")(case.nxp, case.nyp, case.nzp, nx, ny, nz, case.ntheta,
                                               _fp(A), _fp(wav), _ptrs(mm), _ptrs(out))
    assert rc == 0
    return out


def synt_seismic_local(case, m, rel_thick, dz, shift=None, gain=None, nx=None, ny=None, nz=None):
    """Synthetic seismic with each trace's local wavelet (relative
    thickness stretch, local shift and gain): the reference's trace loop on
    its own FFTW (oracle/_ref only).  rel_thick [nyp, nxp] float64; shift /
    gain [ntheta, ny, nx] float32 or None."""
    lib = _load("ref")
    nx = case.nxp if nx is None else nx
    ny = case.nyp if ny is None else ny
    nz = case.nz if nz is None else nz
    mm = [np.ascontiguousarray(g, dtype=np.float32) for g in m]
    out = [np.zeros_like(mm[0]) for _ in range(case.ntheta)]
    A = np.ascontiguousarray(case.A, dtype=np.float32)
    wav = np.ascontiguousarray(case.wavelet, dtype=np.float32)
    rt = np.ascontiguousarray(rel_thick, dtype=np.float64)
    sh = None if shift is None else np.ascontiguousarray(shift, dtype=np.float32)
    ga = None if gain is None else np.ascontiguousarray(gain, dtype=np.float32)
    rc = lib.ref_synt_seismic_local(case.nxp, case.nyp, case.nzp, nx, ny, nz, case.ntheta, _fp(A), _fp(wav),
                                    _ptrs(mm), _dp(rt), float(dz), _fp(sh) if sh is not None else None,
                                    _fp(ga) if ga is not None else None, _ptrs(out))
    assert rc == 0
    return out


def circ_corr_t(prior_corr_t, low_int_cut, nzp, which="orc"):
    """computeCircCorrT + makeCircCorrTPosDef."""
    lib = _load(which)
    pc = np.ascontiguousarray(prior_corr_t, dtype=np.float32)
    out = np.zeros(nzp, np.float32)
    rc = getattr(lib, f"{which}_circ_corr_t")(_fp(pc), pc.size, low_int_cut, nzp, _fp(out))
    assert rc == 0
    return out


def fill_prior_cov(nxp, nyp, nzp, corr_xy, circ, grad_i, grad_j, var0):
    """fillInParamCorr x var0 for the six covariance grids (restatement)."""
    lib = _load("orc")
    cxy = np.ascontiguousarray(corr_xy, dtype=np.float32)
    cc = np.ascontiguousarray(circ, dtype=np.float32)
    v0 = np.ascontiguousarray(var0, dtype=np.float64)
    out = [np.zeros((nzp, nyp, 2 * (nxp // 2 + 1)), np.float32) for _ in range(6)]
    assert lib.orc_fill_prior_cov(nxp, nyp, nzp, _fp(cxy), _fp(cc), grad_i, grad_j, _dp(v0),
                                  _ptrs(out)) == 0
    return out


def fill_err_corr(nxp, nyp, nzp, corr_xy, grad_i, grad_j):
    """fillInErrCorr (restatement)."""
    lib = _load("orc")
    cxy = np.ascontiguousarray(corr_xy, dtype=np.float32)
    out = np.zeros((nzp, nyp, 2 * (nxp // 2 + 1)), np.float32)
    assert lib.orc_fill_err_corr(nxp, nyp, nzp, _fp(cxy), grad_i, grad_j, _fp(out)) == 0
    return out


def divide_data(case, data, cov_col, rel_thick, nx, ny, dz, shift=None, gain=None, which="orc"):
    """Crava::divideDataByScaleWavelet without interpolateSeismic: returns
    new data grids (the inputs are not changed)."""
    keep = []
    p, keep = make_params(case, keep)
    out = [np.ascontiguousarray(g, dtype=np.float32).copy() for g in data]
    col = np.ascontiguousarray(cov_col, dtype=np.float32)
    rt = np.ascontiguousarray(rel_thick, dtype=np.float64)
    sh = np.ascontiguousarray(shift, dtype=np.float32) if shift is not None else None
    gn = np.ascontiguousarray(gain, dtype=np.float32) if gain is not None else None
    rc = getattr(_load(which), f"{which}_divide_data")(
        C.byref(p), _ptrs(out), _fp(col), _dp(rt), nx, ny, dz,
        _fp(sh) if sh is not None else None, _fp(gn) if gn is not None else None)
    assert rc == 0
    return out


def multiply_data(case, data, rel_thick, nx, ny, dz, shift=None, gain=None, which="orc"):
    """multiplyDataByScaleWaveletAndWriteToFile before the write, on
    time-domain residual grids (restatement); returns new grids."""
    keep = []
    p, keep = make_params(case, keep)
    out = [np.ascontiguousarray(g, dtype=np.float32).copy() for g in data]
    rt = np.ascontiguousarray(rel_thick, dtype=np.float64)
    sh = np.ascontiguousarray(shift, dtype=np.float32) if shift is not None else None
    gn = np.ascontiguousarray(gain, dtype=np.float32) if gain is not None else None
    assert getattr(_load(which), f"{which}_multiply_data")(
        C.byref(p), _ptrs(out), _dp(rt), nx, ny, dz, _fp(sh) if sh is not None else None,
        _fp(gn) if gn is not None else None) == 0
    return out


def interpolate_seismic(grid, nxp, nyp, nzp, nx, ny, nz, energy_threshold):
    """FFTGrid::interpolateSeismic + extrapolateSeismic (restatement);
    returns (new grid, traces interpolated, of which zero energy)."""
    lib = _load("orc")
    g = np.ascontiguousarray(grid, dtype=np.float32).copy()
    ni, n0 = C.c_int(0), C.c_int(0)
    assert lib.orc_interpolate_seismic(_fp(g), nxp, nyp, nzp, nx, ny, nz, energy_threshold,
                                       C.byref(ni), C.byref(n0)) == 0
    return g, ni.value, n0.value


STATE_KEYS = ("ms", "md", "ss", "dd", "sd")  # 3, 3, 6, 6, 9 spectra


def _state_ptrs(state):
    return [_ptrs(state[k]) for k in STATE_KEYS]


def state4d_merge(state, mu, cov, which="orc"):
    """State4D::merge / mergeCov into mu (3, or None) and cov (6, posterior
    order); spectra as float32 arrays of interleaved complex values."""
    lib = _load(which)
    n = state["ms"][0].size // 2
    getattr(lib, f"{which}_state4d_merge")(n, *_state_ptrs(state),
                                           _ptrs(mu) if mu is not None else None, _ptrs(cov))


def state4d_split(state, mu, cov, which="orc"):
    """State4D::split, in place on state; returns the shortcut bins."""
    lib = _load(which)
    n = state["ms"][0].size // 2
    return int(getattr(lib, f"{which}_state4d_split")(n, *_state_ptrs(state), _ptrs(mu), _ptrs(cov)))


def state4d_evolve(state, E, cm, cc, lam, zero_scale):
    """State4D::evolve (restatement), in place on state."""
    lib = _load("orc")
    n = state["ms"][0].size // 2
    E, cm, cc = (np.ascontiguousarray(x, dtype=np.float64).reshape(-1) for x in (E, cm, cc))
    lib.orc_state4d_evolve(n, *_state_ptrs(state), _dp(E), _dp(cm), _dp(cc), _fp(lam), zero_scale)


def fill_gen_exp_corr(nxp, nyp, nzp, rx, ry, rz, grad_i, grad_j):
    """FFTGrid::fillInGenExpCorr (restatement)."""
    lib = _load("orc")
    out = np.zeros((nzp, nyp, 2 * (nxp // 2 + 1)), np.float32)
    assert lib.orc_fill_gen_exp_corr(nxp, nyp, nzp, rx, ry, rz, grad_i, grad_j, _fp(out)) == 0
    return out


def complex_view(g, nxp):
    """[nzp, nyp, rnxp] float32 -> [nzp, nyp, cnxp] complex64 view."""
    return g.view(np.complex64)[..., : nxp // 2 + 1]
