"""Python binding of the C ABI (include/crava_gpu.h) over ctypes.

PyTorch provides device memory and streams; every computation runs in the
in-tree CUDA library crava_b200/lib/libcrava_gpu.so.  There is no CPU path:
if the library or a CUDA device is missing, the calls raise.

The classes mirror the reference interface this path replaces:
  FFTGrid  -- a padded grid in HBM with fftInPlace / invFFTInPlace
              (src/fftgrid.h:110-143 of the reference);
  Crava    -- computePostMeanResidAndFFTCov and simulate on a set of grids
              (src/crava.h:35-79).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libcrava_gpu.so")

MAX_THETA = 8
OK = 0
STATUS = {0: "ok", 1: "invalid argument", 2: "allocation failed", 3: "CUDA error",
          4: "device wait timed out", 5: "call out of order", 6: "no CUDA device"}
DATA, PARAMETER, COVARIANCE = 1, 2, 3
FP64, MIXED, FP32 = 0, 1, 2

F32P = C.POINTER(C.c_float)
F64P = C.POINTER(C.c_double)


class Params(C.Structure):
    _fields_ = [
        ("nxp", C.c_int), ("nyp", C.c_int), ("nzp", C.c_int), ("ntheta", C.c_int),
        ("nz", C.c_int), ("precision", C.c_int),
        ("lz", C.c_double), ("min_rel_thick", C.c_double),
        ("low_cut", C.c_float), ("high_cut", C.c_float), ("wnc", C.c_float),
        ("thickness_mode", C.c_int),
        ("wavelet", F32P), ("wavelet_norm", F32P), ("A", F32P),
        ("theta_cov", F64P), ("var0", F64P),
    ]


class Grids(C.Structure):
    _fields_ = [("mu", C.c_void_p * 3), ("data", C.c_void_p * MAX_THETA),
                ("cov", C.c_void_p * 6), ("err_corr", C.c_void_p)]


class KernelProfile(C.Structure):
    _fields_ = [("name", C.c_char * 32), ("launches", C.c_longlong), ("total_ms", C.c_double),
                ("bytes_per_launch", C.c_double)]


class State4DGrids(C.Structure):
    """crava_gpu_state4d: the static/dynamic time-lapse state (State4D)."""
    _fields_ = [("mu_static", C.c_void_p * 3), ("mu_dynamic", C.c_void_p * 3),
                ("cov_ss", C.c_void_p * 6), ("cov_dd", C.c_void_p * 6), ("cov_sd", C.c_void_p * 9)]


class Stats(C.Structure):
    _fields_ = [("chol_fail_bins", C.c_longlong), ("nonfinite_bins", C.c_longlong),
                ("ms_forward", C.c_float), ("ms_solve", C.c_float),
                ("ms_inverse", C.c_float), ("ms_total", C.c_float), ("refined_bins", C.c_longlong),
                ("tile_wait_timeouts", C.c_longlong)]


class Tuning(C.Structure):
    _fields_ = [("cols_y_tile", C.c_int), ("cols_z_tile", C.c_int), ("fused", C.c_int),
                ("ms", C.c_float), ("lanes", C.c_int), ("rows_x", C.c_int), ("kappa_refine", C.c_float),
                ("xy_fused", C.c_int), ("solve_shape", C.c_int)]


class GridHeader(C.Structure):
    _fields_ = [("x0", C.c_double), ("y0", C.c_double), ("dx", C.c_double), ("dy", C.c_double),
                ("nx", C.c_int), ("ny", C.c_int), ("il0", C.c_double), ("xl0", C.c_double),
                ("il_step_x", C.c_double), ("il_step_y", C.c_double), ("xl_step_x", C.c_double),
                ("xl_step_y", C.c_double), ("angle", C.c_double)]


class Vintage(C.Structure):
    _fields_ = [("ctx", C.c_void_p), ("inp", Grids), ("out", Grids), ("precision", C.c_int),
                ("nsim", C.c_int), ("seed", C.c_uint64), ("first_index", C.c_uint64),
                ("sim_out", C.POINTER(C.c_void_p))]


BATCH_AUTOTUNE, BATCH_NO_GRAPH = 1, 2

SYMBOLS = {
    "crava_gpu_create": ([C.POINTER(Params), C.c_int, C.c_void_p, C.POINTER(C.c_void_p)], C.c_int),
    "crava_gpu_destroy": ([C.c_void_p], C.c_int),
    "crava_gpu_status_string": ([C.c_int], C.c_char_p),
    "crava_gpu_fft_r2c": ([C.c_void_p, C.c_void_p, C.c_int], C.c_int),
    "crava_gpu_fft_c2r": ([C.c_void_p, C.c_void_p, C.c_int], C.c_int),
    "crava_gpu_posterior": ([C.c_void_p, C.POINTER(Grids), C.c_int], C.c_int),
    "crava_gpu_posterior_unit": ([C.c_void_p, C.POINTER(Grids), C.c_int], C.c_int),
    "crava_gpu_posterior_unit_oop": ([C.c_void_p, C.POINTER(Grids), C.POINTER(Grids), C.c_int], C.c_int),
    "crava_gpu_set_fused": ([C.c_void_p, C.c_int], C.c_int),
    "crava_gpu_fused_available": ([C.c_void_p, C.c_int], C.c_int),
    "crava_gpu_set_profiling": ([C.c_void_p, C.c_int], C.c_int),
    "crava_gpu_get_profile": ([C.c_void_p, C.POINTER(KernelProfile), C.c_int, C.POINTER(C.c_int)], C.c_int),
    "crava_gpu_posterior_unit_host": ([C.c_void_p, C.POINTER(Grids), C.c_int], C.c_int),
    "crava_gpu_host_register": ([C.c_void_p, C.c_uint64], C.c_int),
    "crava_gpu_host_unregister": ([C.c_void_p], C.c_int),
    "crava_gpu_noise_fill": ([C.c_void_p, C.c_void_p, C.c_uint64, C.c_uint64], C.c_int),
    "crava_gpu_sim_filter": ([C.c_void_p, C.c_void_p * 6, C.c_void_p * 3], C.c_int),
    "crava_gpu_simulate": ([C.c_void_p, C.c_void_p * 6, C.c_void_p * 3, C.c_uint64, C.c_int,
                            C.c_int, C.POINTER(C.c_void_p)], C.c_int),
    "crava_gpu_get_stats": ([C.c_void_p, C.POINTER(Stats)], C.c_int),
    "crava_gpu_kz_tables": ([C.c_void_p, F32P, F32P, F32P, F32P, C.POINTER(C.c_int)], C.c_int),
    "crava_gpu_set_kz_tables": ([C.c_void_p, F32P, F32P, F32P, F32P, C.POINTER(C.c_int)], C.c_int),
    "crava_gpu_launch_count": ([], C.c_longlong),
    "crava_gpu_get_tuning": ([C.c_void_p, C.POINTER(Tuning)], C.c_int),
    "crava_gpu_set_tuning": ([C.c_void_p, C.POINTER(Tuning)], C.c_int),
    "crava_gpu_autotune": ([C.c_void_p, C.POINTER(Grids), C.POINTER(Grids), C.c_int, C.c_int,
                            C.POINTER(Tuning)], C.c_int),
    "crava_gpu_batch_create": ([C.POINTER(Vintage), C.c_int, C.c_int, C.c_void_p,
                                C.POINTER(C.c_void_p)], C.c_int),
    "crava_gpu_batch_run": ([C.c_void_p], C.c_int),
    "crava_gpu_batch_sync": ([C.c_void_p], C.c_int),
    "crava_gpu_batch_destroy": ([C.c_void_p], C.c_int),
    "crava_gpu_loglik_grad": ([C.c_void_p, C.POINTER(Grids), F64P, F64P, F64P, F64P, F64P, F64P, F64P,
                               C.POINTER(C.c_longlong)], C.c_int),
    "crava_gpu_synt_seismic": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int,
                                C.POINTER(C.c_void_p)], C.c_int),
    "crava_gpu_synt_seismic_local": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, F64P,
                                      C.c_float, F32P, F32P, C.POINTER(C.c_void_p)], C.c_int),
    "crava_gpu_circ_corr_t": ([F32P, C.c_int, C.c_int, C.c_int, F32P], C.c_int),
    "crava_gpu_fill_prior_cov": ([C.c_void_p, F32P, F32P, C.c_float, C.c_float, C.POINTER(C.c_void_p)],
                                 C.c_int),
    "crava_gpu_fill_err_corr": ([C.c_void_p, F32P, C.c_float, C.c_float, C.c_void_p], C.c_int),
    "crava_gpu_posterior_unit_host_async": ([C.c_void_p, C.POINTER(Grids), C.POINTER(Grids), C.c_int],
                                            C.c_int),
    "crava_gpu_host_wait": ([C.c_void_p], C.c_int),
    "crava_gpu_crava_file_write": ([C.c_void_p, C.c_char_p, C.c_void_p, C.POINTER(GridHeader)], C.c_int),
    "crava_gpu_crava_file_read": ([C.c_void_p, C.c_char_p, C.c_void_p, C.POINTER(GridHeader)], C.c_int),
    "crava_gpu_state4d_merge": ([C.c_void_p, C.POINTER(State4DGrids), C.POINTER(C.c_void_p),
                                 C.POINTER(C.c_void_p)], C.c_int),
    "crava_gpu_state4d_split": ([C.c_void_p, C.POINTER(State4DGrids), C.POINTER(C.c_void_p),
                                 C.POINTER(C.c_void_p), C.POINTER(C.c_longlong)], C.c_int),
    "crava_gpu_fill_gen_exp_corr": ([C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_float,
                                     C.c_float, C.c_void_p], C.c_int),
    "crava_gpu_state4d_evolve": ([C.c_void_p, C.POINTER(State4DGrids), F64P, F64P, F64P, C.c_void_p],
                                 C.c_int),
    "crava_gpu_state4d_advance_time": ([C.c_void_p, C.POINTER(State4DGrids), C.c_int, C.c_int, C.c_int,
                                        F64P, F64P, F64P, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p),
                                        C.c_void_p, C.POINTER(C.c_longlong)], C.c_int),
    "crava_gpu_divide_data_by_scale_wavelet": ([C.c_void_p, C.POINTER(C.c_void_p), C.c_void_p, F64P, C.c_int,
                                                C.c_int, C.c_float, F32P, F32P], C.c_int),
    "crava_gpu_multiply_data_by_scale_wavelet": ([C.c_void_p, C.POINTER(C.c_void_p), F64P, C.c_int, C.c_int,
                                                  C.c_float, F32P, F32P], C.c_int),
    "crava_gpu_interpolate_seismic": ([C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_float,
                                       C.POINTER(C.c_int), C.POINTER(C.c_int)], C.c_int),
    "crava_gpu_fft_xy": ([C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int], C.c_int),
    "crava_gpu_fft_z": ([C.c_void_p, C.c_void_p, C.c_int], C.c_int),
    "crava_gpu_posterior_noalloc": ([C.POINTER(Params), C.POINTER(Grids), C.c_int, C.c_void_p,
                                     C.POINTER(Stats)], C.c_int),
}

_lib = None


class CravaGpuError(RuntimeError):
    pass


def load_library(path: str = LIB_PATH):
    """Loads the CUDA library; raises if it is missing (no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise CravaGpuError(f"CUDA library not built: {path} (run crava_b200/build.py)")
    lib = C.CDLL(path)
    for name, (args, res) in SYMBOLS.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res
    _lib = lib
    return lib


def check(rc: int, what: str = "") -> None:
    if rc != OK:
        msg = load_library().crava_gpu_status_string(rc).decode()
        raise CravaGpuError(f"{what}: status {rc} ({msg})")


def launch_count() -> int:
    return int(load_library().crava_gpu_launch_count())


def _ptr(t):
    return C.c_void_p(t.data_ptr())


class Context:
    """A crava_gpu_ctx bound to one device and one CUDA stream."""

    def __init__(self, case, device: int = 0, stream=None, precision: int = MIXED,
                 wavelet_norm=None):
        import torch

        lib = load_library()
        self._keep = []
        wav = np.ascontiguousarray(case.wavelet, dtype=np.float32)
        A = np.ascontiguousarray(case.A, dtype=np.float32)
        th = np.ascontiguousarray(case.theta_cov, dtype=np.float64)
        v0 = np.ascontiguousarray(case.var0, dtype=np.float64)
        self._keep += [wav, A, th, v0]
        wn = None
        if wavelet_norm is not None:
            wn = np.ascontiguousarray(wavelet_norm, dtype=np.float32)
            self._keep.append(wn)
        self.params = Params(case.nxp, case.nyp, case.nzp, case.ntheta, case.nz, precision,
                             case.lz, case.min_rel_thick, case.low_cut, case.high_cut, case.wnc,
                             int(getattr(case, "thickness_mode", 0)), wav.ctypes.data_as(F32P),
                             wn.ctypes.data_as(F32P) if wn is not None else None,
                             A.ctypes.data_as(F32P), th.ctypes.data_as(F64P),
                             v0.ctypes.data_as(F64P))
        self.case = case
        self.device = device
        self.stream = stream if stream is not None else torch.cuda.current_stream(device)
        self.precision = precision
        h = C.c_void_p()
        check(lib.crava_gpu_create(C.byref(self.params), device, C.c_void_p(self.stream.cuda_stream),
                                   C.byref(h)), "crava_gpu_create")
        self.handle = h
        self.lib = lib

    def close(self):
        if getattr(self, "handle", None):
            self.lib.crava_gpu_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- grids
    def grids(self, mu, data, cov, err):
        g = Grids()
        for q in range(3):
            g.mu[q] = mu[q].data_ptr()
        for l in range(len(data)):
            g.data[l] = data[l].data_ptr()
        for t in range(6):
            g.cov[t] = cov[t].data_ptr()
        g.err_corr = err.data_ptr()
        return g

    def fft_r2c(self, grid, grid_type):
        check(self.lib.crava_gpu_fft_r2c(self.handle, _ptr(grid), grid_type), "fft_r2c")

    def fft_c2r(self, grid, grid_type):
        check(self.lib.crava_gpu_fft_c2r(self.handle, _ptr(grid), grid_type), "fft_c2r")

    def fft_xy(self, grid, direction, grid_type, nzp_full=None):
        """The x and y passes only (-1 forward, +1 inverse), scaled as the
        whole grid of nzp_full planes (crava_gpu_fft_xy): one z slab of a
        grid split over GPUs."""
        nz = self.case.nzp if nzp_full is None else nzp_full
        check(self.lib.crava_gpu_fft_xy(self.handle, _ptr(grid), direction, grid_type, nz), "fft_xy")

    def fft_z(self, grid, direction):
        """The unscaled z pass only (crava_gpu_fft_z): one column shard."""
        check(self.lib.crava_gpu_fft_z(self.handle, _ptr(grid), direction), "fft_z")

    def posterior(self, mu, data, cov, err, precision=None):
        g = self.grids(mu, data, cov, err)
        p = self.precision if precision is None else precision
        check(self.lib.crava_gpu_posterior(self.handle, C.byref(g), p), "posterior")

    def posterior_unit(self, mu, data, cov, err, precision=None):
        g = self.grids(mu, data, cov, err)
        p = self.precision if precision is None else precision
        check(self.lib.crava_gpu_posterior_unit(self.handle, C.byref(g), p), "posterior_unit")

    def posterior_unit_oop(self, src, dst, precision=None):
        """src, dst: (mu, data, cov, err) tuples of device tensors."""
        gi = self.grids(*src)
        go = self.grids(*dst)
        p = self.precision if precision is None else precision
        check(self.lib.crava_gpu_posterior_unit_oop(self.handle, C.byref(gi), C.byref(go), p),
              "posterior_unit_oop")

    def tuning(self) -> Tuning:
        t = Tuning()
        check(self.lib.crava_gpu_get_tuning(self.handle, C.byref(t)), "get_tuning")
        return t

    def set_tuning(self, cols_y_tile=-1, cols_z_tile=-1, fused=0, lanes=3, rows_x=-1, kappa_refine=None,
                   xy_fused=None, solve_shape=None):
        cur = self.tuning()
        if kappa_refine is None:
            kappa_refine = cur.kappa_refine
        if xy_fused is None:
            xy_fused = cur.xy_fused
        if solve_shape is None:
            solve_shape = cur.solve_shape
        t = Tuning(cols_y_tile, cols_z_tile, fused, 0.0, lanes, rows_x, kappa_refine, xy_fused, solve_shape)
        check(self.lib.crava_gpu_set_tuning(self.handle, C.byref(t)), "set_tuning")

    def autotune(self, src, dst, precision=None, reps=2) -> Tuning:
        """Times every launch-shape candidate on the out-of-place unit
        src -> dst and keeps the fastest (synchronous)."""
        gi, go = self.grids(*src), self.grids(*dst)
        p = self.precision if precision is None else precision
        t = Tuning()
        check(self.lib.crava_gpu_autotune(self.handle, C.byref(gi), C.byref(go), p, reps, C.byref(t)),
              "autotune")
        return t

    def loglik_grad(self, mu, data, cov, err, wavelet_scale=None, noise_var=None, wavelet_spec=None):
        """Log marginal likelihood of the transformed data and its gradients
        (crava_gpu_loglik_grad).  wavelet_spec / the returned spectrum
        gradient: complex [nzp/2+1, ntheta].  Returns (L, g_scale, g_noise,
        g_spec, failed_bins)."""
        nt, cn = self.case.ntheta, self.case.nzp // 2 + 1
        g = self.grids(mu, data, cov, err)
        f64 = lambda a: None if a is None else np.ascontiguousarray(a, dtype=np.float64)
        sc, nv = f64(wavelet_scale), f64(noise_var)
        sp = None
        if wavelet_spec is not None:
            w = np.asarray(wavelet_spec)
            sp = np.ascontiguousarray(np.stack([w.real, w.imag], -1), dtype=np.float64) \
                if np.iscomplexobj(w) else f64(w)
            assert sp.size == cn * nt * 2
        ptr = lambda a: a.ctypes.data_as(F64P) if a is not None else None
        L = C.c_double(0.0)
        gs, gv = np.zeros(nt), np.zeros(nt)
        gw = np.zeros((cn, nt, 2))
        nf = C.c_longlong(0)
        check(self.lib.crava_gpu_loglik_grad(self.handle, C.byref(g), ptr(sc), ptr(nv), ptr(sp),
                                             C.byref(L), ptr(gs), ptr(gv), ptr(gw), C.byref(nf)),
              "loglik_grad")
        return L.value, gs, gv, gw[..., 0] + 1j * gw[..., 1], nf.value

    def fill_prior_cov(self, corr_xy, circ_corr_t, grad_i, grad_j, cov):
        """The six prior covariance grids (SeismicParametersHolder::
        initializeCorrelations) written on the device into cov."""
        cxy = np.ascontiguousarray(corr_xy, dtype=np.float32)
        cc = np.ascontiguousarray(circ_corr_t, dtype=np.float32)
        assert cxy.size == self.case.nxp * self.case.nyp and cc.size == self.case.nzp
        arr = (C.c_void_p * 6)(*[g.data_ptr() for g in cov])
        check(self.lib.crava_gpu_fill_prior_cov(self.handle, cxy.ctypes.data_as(F32P), cc.ctypes.data_as(F32P),
                                                grad_i, grad_j, arr), "fill_prior_cov")

    def fill_err_corr(self, corr_xy, grad_i, grad_j, err):
        """The noise correlation grid (FFTGrid::fillInErrCorr) on the device."""
        cxy = np.ascontiguousarray(corr_xy, dtype=np.float32)
        assert cxy.size == self.case.nxp * self.case.nyp
        check(self.lib.crava_gpu_fill_err_corr(self.handle, cxy.ctypes.data_as(F32P), grad_i, grad_j,
                                               _ptr(err)), "fill_err_corr")

    def divide_data_by_scale_wavelet(self, data, cov_alpha, rel_thick, nx, ny, dz, shift=None, gain=None):
        """Crava::divideDataByScaleWavelet (without interpolateSeismic) on
        the device data grids, in place.  cov_alpha: the real-domain prior
        covAlpha device grid; rel_thick: [nyp, nxp]; shift, gain:
        [ntheta, ny, nx] or None."""
        rt = np.ascontiguousarray(rel_thick, dtype=np.float64)
        assert rt.size == self.case.nxp * self.case.nyp
        arr = (C.c_void_p * len(data))(*[g.data_ptr() for g in data])
        sh = np.ascontiguousarray(shift, dtype=np.float32) if shift is not None else None
        gn = np.ascontiguousarray(gain, dtype=np.float32) if gain is not None else None
        for x in (sh, gn):
            assert x is None or x.size == len(data) * nx * ny
        check(self.lib.crava_gpu_divide_data_by_scale_wavelet(
            self.handle, arr, _ptr(cov_alpha), rt.ctypes.data_as(F64P), nx, ny, dz,
            sh.ctypes.data_as(F32P) if sh is not None else None,
            gn.ctypes.data_as(F32P) if gn is not None else None), "divide_data_by_scale_wavelet")

    def multiply_data_by_scale_wavelet(self, resid, rel_thick, nx, ny, dz, shift=None, gain=None):
        """Crava::multiplyDataByScaleWaveletAndWriteToFile without the file
        write: transformed residual grids back to the time domain, each
        simbox trace times its local wavelet's conjugate spectrum."""
        rt = np.ascontiguousarray(rel_thick, dtype=np.float64)
        assert rt.size == self.case.nxp * self.case.nyp
        arr = (C.c_void_p * len(resid))(*[g.data_ptr() for g in resid])
        sh = np.ascontiguousarray(shift, dtype=np.float32) if shift is not None else None
        gn = np.ascontiguousarray(gain, dtype=np.float32) if gain is not None else None
        check(self.lib.crava_gpu_multiply_data_by_scale_wavelet(
            self.handle, arr, rt.ctypes.data_as(F64P), nx, ny, dz,
            sh.ctypes.data_as(F32P) if sh is not None else None,
            gn.ctypes.data_as(F32P) if gn is not None else None), "multiply_data_by_scale_wavelet")

    def interpolate_seismic(self, grid, nx, ny, energy_threshold):
        """FFTGrid::interpolateSeismic on a device data grid, in place;
        returns (traces interpolated, of which zero energy)."""
        ni, n0 = C.c_int(0), C.c_int(0)
        check(self.lib.crava_gpu_interpolate_seismic(self.handle, _ptr(grid), nx, ny, energy_threshold,
                                                     C.byref(ni), C.byref(n0)), "interpolate_seismic")
        return ni.value, n0.value

    # ---- time-lapse state (State4D, src/state4d.cpp) -------------------
    @staticmethod
    def _state(state) -> State4DGrids:
        """state: dict with 'ms', 'md' (3 each), 'ss', 'dd' (6 each) and 'sd'
        (9) device grids holding Fourier-domain spectra."""
        st = State4DGrids()
        for key, field, n in (("ms", "mu_static", 3), ("md", "mu_dynamic", 3), ("ss", "cov_ss", 6),
                              ("dd", "cov_dd", 6), ("sd", "cov_sd", 9)):
            assert len(state[key]) == n, key
            setattr(st, field, (C.c_void_p * n)(*[g.data_ptr() for g in state[key]]))
        return st

    def state4d_merge(self, state, mu, cov):
        """State4D::merge (mu None: mergeCov) into Fourier-domain grids."""
        st = self._state(state)
        m = (C.c_void_p * 3)(*[g.data_ptr() for g in mu]) if mu is not None else None
        c = (C.c_void_p * 6)(*[g.data_ptr() for g in cov])
        check(self.lib.crava_gpu_state4d_merge(self.handle, C.byref(st), m, c), "state4d_merge")

    def state4d_split(self, state, mu, cov) -> int:
        """State4D::split of the inverted current state; returns the bins
        whose Cholesky failed (prior kept)."""
        st = self._state(state)
        m = (C.c_void_p * 3)(*[g.data_ptr() for g in mu])
        c = (C.c_void_p * 6)(*[g.data_ptr() for g in cov])
        n = C.c_longlong(0)
        check(self.lib.crava_gpu_state4d_split(self.handle, C.byref(st), m, c, C.byref(n)), "state4d_split")
        return n.value

    def fill_gen_exp_corr(self, rx, ry, rz, grad_i, grad_j, grid):
        """FFTGrid::fillInGenExpCorr on the device."""
        check(self.lib.crava_gpu_fill_gen_exp_corr(self.handle, rx, ry, rz, grad_i, grad_j, _ptr(grid)),
              "fill_gen_exp_corr")

    def state4d_evolve(self, state, evolution, mean_correction, cov_correction, lam):
        """State4D::evolve with the transformed time-increment correlation."""
        st = self._state(state)
        E, cm, cc = (np.ascontiguousarray(x, dtype=np.float64).reshape(-1)
                     for x in (evolution, mean_correction, cov_correction))
        assert E.size == 36 and cm.size == 6 and cc.size == 36
        check(self.lib.crava_gpu_state4d_evolve(self.handle, C.byref(st), E.ctypes.data_as(F64P),
                                                cm.ctypes.data_as(F64P), cc.ctypes.data_as(F64P), _ptr(lam)),
              "state4d_evolve")

    def advance_time(self, state, time_step, nx, ny, evolution, mean_correction, cov_correction,
                     mu, cov, lambda_work) -> int:
        """ModelGeneral::advanceTime: split, evolve, merge, back to the time
        domain.  Returns the split's shortcut bins."""
        st = self._state(state)
        E, cm, cc = (np.ascontiguousarray(x, dtype=np.float64).reshape(-1)
                     for x in (evolution, mean_correction, cov_correction))
        assert E.size == 36 and cm.size == 6 and cc.size == 36
        m = (C.c_void_p * 3)(*[g.data_ptr() for g in mu])
        c = (C.c_void_p * 6)(*[g.data_ptr() for g in cov])
        n = C.c_longlong(0)
        check(self.lib.crava_gpu_state4d_advance_time(
            self.handle, C.byref(st), time_step, nx, ny, E.ctypes.data_as(F64P), cm.ctypes.data_as(F64P),
            cc.ctypes.data_as(F64P), m, c, _ptr(lambda_work), C.byref(n)), "advance_time")
        return n.value

    def write_crava_file(self, path, grid, header: "GridHeader"):
        """FFTGrid::writeCravaFile of a device grid."""
        check(self.lib.crava_gpu_crava_file_write(self.handle, os.fsencode(path), _ptr(grid), C.byref(header)),
              "crava_file_write")

    def read_crava_file(self, path, grid) -> "GridHeader":
        """FFTGrid::readCravaFile into a device grid; returns the header."""
        h = GridHeader()
        check(self.lib.crava_gpu_crava_file_read(self.handle, os.fsencode(path), _ptr(grid), C.byref(h)),
              "crava_file_read")
        return h

    def synt_seismic(self, alpha, beta, rho, outs, nx=0, ny=0):
        """Synthetic seismic of the real parameter grids into outs (one real
        grid per angle), Crava::computeSyntSeismic."""
        arr = (C.c_void_p * len(outs))(*[o.data_ptr() for o in outs])
        check(self.lib.crava_gpu_synt_seismic(self.handle, _ptr(alpha), _ptr(beta), _ptr(rho), nx, ny, arr),
              "synt_seismic")

    def synt_seismic_local(self, alpha, beta, rho, outs, rel_thick, dz, shift=None, gain=None, nx=0, ny=0):
        """Synthetic seismic with every simbox trace's local wavelet
        (stretch rel_thick [nyp, nxp], local shift / gain [ntheta, ny, nx])."""
        rt = np.ascontiguousarray(rel_thick, dtype=np.float64)
        assert rt.size == self.case.nxp * self.case.nyp
        sh = np.ascontiguousarray(shift, dtype=np.float32) if shift is not None else None
        gn = np.ascontiguousarray(gain, dtype=np.float32) if gain is not None else None
        arr = (C.c_void_p * len(outs))(*[o.data_ptr() for o in outs])
        check(self.lib.crava_gpu_synt_seismic_local(
            self.handle, _ptr(alpha), _ptr(beta), _ptr(rho), nx, ny, rt.ctypes.data_as(F64P), dz,
            sh.ctypes.data_as(F32P) if sh is not None else None,
            gn.ctypes.data_as(F32P) if gn is not None else None, arr), "synt_seismic_local")

    def set_fused(self, enable=True):
        check(self.lib.crava_gpu_set_fused(self.handle, int(bool(enable))), "set_fused")

    def fused_available(self, precision=None):
        p = self.precision if precision is None else precision
        return bool(self.lib.crava_gpu_fused_available(self.handle, p))

    def set_profiling(self, enable=True):
        check(self.lib.crava_gpu_set_profiling(self.handle, int(bool(enable))), "set_profiling")

    def profile(self):
        """{name: (launches, total_ms, bytes_per_launch)}; resets the counters."""
        arr = (KernelProfile * 16)()
        n = C.c_int(0)
        check(self.lib.crava_gpu_get_profile(self.handle, arr, 16, C.byref(n)), "get_profile")
        return {arr[i].name.decode(): (arr[i].launches, arr[i].total_ms, arr[i].bytes_per_launch)
                for i in range(min(n.value, 16))}

    def posterior_unit_host(self, mu, data, cov, err, precision=None):
        """Host tensors (CPU, ideally pinned); synchronous."""
        g = self.grids(mu, data, cov, err)
        p = self.precision if precision is None else precision
        check(self.lib.crava_gpu_posterior_unit_host(self.handle, C.byref(g), p), "posterior_unit_host")

    def posterior_unit_host_async(self, src, dst, precision=None):
        """src, dst: (mu, data, cov, err) tuples of host tensors (pinned);
        returns once enqueued; call host_wait() before touching them."""
        gi, go = self.grids(*src), self.grids(*dst)
        p = self.precision if precision is None else precision
        check(self.lib.crava_gpu_posterior_unit_host_async(self.handle, C.byref(gi), C.byref(go), p),
              "posterior_unit_host_async")

    def host_wait(self):
        check(self.lib.crava_gpu_host_wait(self.handle), "host_wait")

    def noise_fill(self, grid, seed, stream_id):
        check(self.lib.crava_gpu_noise_fill(self.handle, _ptr(grid), seed, stream_id), "noise_fill")

    def sim_filter(self, cov, seeds):
        cv = (C.c_void_p * 6)(*[c.data_ptr() for c in cov])
        sd = (C.c_void_p * 3)(*[s.data_ptr() for s in seeds])
        check(self.lib.crava_gpu_sim_filter(self.handle, cv, sd), "sim_filter")

    def simulate(self, cov, post_mean, seed, first_index, outs):
        """outs: list of 3*count real grids (device)."""
        cv = (C.c_void_p * 6)(*[c.data_ptr() for c in cov])
        pm = (C.c_void_p * 3)(*[m.data_ptr() for m in post_mean])
        count = len(outs) // 3
        arr = (C.c_void_p * max(1, len(outs)))(*[o.data_ptr() for o in outs])
        check(self.lib.crava_gpu_simulate(self.handle, cv, pm, seed, first_index, count, arr), "simulate")

    def stats(self) -> Stats:
        s = Stats()
        check(self.lib.crava_gpu_get_stats(self.handle, C.byref(s)), "get_stats")
        return s

    def kz_tables(self):
        nzp, nt = self.case.nzp, self.case.ntheta
        n = nzp * nt
        wd = np.zeros(2 * n, np.float32); e1 = np.zeros(2 * n, np.float32)
        e2 = np.zeros(2 * n, np.float32); e3 = np.zeros(n, np.float32)
        inv = np.zeros(nzp, np.int32)
        check(self.lib.crava_gpu_kz_tables(self.handle, wd.ctypes.data_as(F32P), e1.ctypes.data_as(F32P),
                                           e2.ctypes.data_as(F32P), e3.ctypes.data_as(F32P),
                                           inv.ctypes.data_as(C.POINTER(C.c_int))), "kz_tables")
        cpx = lambda a: a.view(np.complex64).reshape(nzp, nt)
        return cpx(wd), cpx(e1), cpx(e2), e3.reshape(nzp, nt), inv

    def set_kz_tables(self, tables):
        wd, e1, e2, e3, inv = tables
        f32 = lambda a: np.ascontiguousarray(a.view(np.float32) if a.dtype == np.complex64 else a,
                                             dtype=np.float32)
        wd, e1, e2, e3 = f32(wd), f32(e1), f32(e2), f32(e3)
        inv = np.ascontiguousarray(inv, dtype=np.int32)
        check(self.lib.crava_gpu_set_kz_tables(self.handle, wd.ctypes.data_as(F32P), e1.ctypes.data_as(F32P),
                                               e2.ctypes.data_as(F32P), e3.ctypes.data_as(F32P),
                                               inv.ctypes.data_as(C.POINTER(C.c_int))), "set_kz_tables")


def circ_corr_t(prior_corr_t, low_int_cut, nzp):
    """Circular temporal prior correlation (crava_gpu_circ_corr_t; host
    computation, no GPU needed)."""
    pc = np.ascontiguousarray(prior_corr_t, dtype=np.float32)
    out = np.zeros(nzp, np.float32)
    check(load_library().crava_gpu_circ_corr_t(pc.ctypes.data_as(F32P), pc.size, low_int_cut, nzp,
                                               out.ctypes.data_as(F32P)), "circ_corr_t")
    return out


class Batch:
    """Vintages (one Context each) inverted and sampled as one CUDA graph
    launch per run.  vintages: dicts with ctx, src and dst ((mu, data, cov,
    err) tuples of device tensors), precision, and optionally nsim, seed,
    first_index and sims (3 * nsim device grids)."""

    def __init__(self, vintages, flags=0, stream=None):
        lib = load_library()
        self.lib = lib
        self._keep = []
        arr = (Vintage * len(vintages))()
        for k, v in enumerate(vintages):
            ctx = v["ctx"]
            nsim = int(v.get("nsim", 0))
            sims = v.get("sims", [])
            assert len(sims) == 3 * nsim
            ptrs = (C.c_void_p * max(1, 3 * nsim))(*[t.data_ptr() for t in sims])
            self._keep += [ptrs, v]
            arr[k].ctx = ctx.handle
            arr[k].inp = ctx.grids(*v["src"])
            arr[k].out = ctx.grids(*v["dst"])
            arr[k].precision = v.get("precision", ctx.precision)
            arr[k].nsim = nsim
            arr[k].seed = int(v.get("seed", 0))
            arr[k].first_index = int(v.get("first_index", 0))
            arr[k].sim_out = C.cast(ptrs, C.POINTER(C.c_void_p)) if nsim else None
        h = C.c_void_p()
        sp = C.c_void_p(stream.cuda_stream) if stream is not None else None
        check(lib.crava_gpu_batch_create(arr, len(vintages), flags, sp, C.byref(h)), "batch_create")
        self.handle = h

    def run(self):
        check(self.lib.crava_gpu_batch_run(self.handle), "batch_run")

    def sync(self):
        check(self.lib.crava_gpu_batch_sync(self.handle), "batch_sync")

    def close(self):
        if getattr(self, "handle", None):
            self.lib.crava_gpu_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def to_device(arr, device=0):
    import torch

    return torch.from_numpy(np.ascontiguousarray(arr, dtype=np.float32)).to(f"cuda:{device}")


def complex_view(t, nxp):
    """[nzp, nyp, rnxp] float tensor/array -> [nzp, nyp, cnxp] complex view."""
    if isinstance(t, np.ndarray):
        return t.view(np.complex64)[..., : nxp // 2 + 1]
    import torch

    return torch.view_as_complex(t.view(*t.shape[:-1], -1, 2))[..., : nxp // 2 + 1]


class FFTGrid:
    """A padded grid resident in HBM -- the device counterpart of the
    reference's FFTGrid (src/fftgrid.h): same layout, same grid types,
    fftInPlace / invFFTInPlace with the same scalings."""

    def __init__(self, ctx: Context, values=None, grid_type: int = PARAMETER):
        import torch

        c = ctx.case
        self.ctx = ctx
        self.nxp, self.nyp, self.nzp = c.nxp, c.nyp, c.nzp
        self.type = grid_type
        shape = (c.nzp, c.nyp, 2 * (c.nxp // 2 + 1))
        if values is None:
            self.t = torch.zeros(shape, dtype=torch.float32, device=f"cuda:{ctx.device}")
        else:
            self.t = to_device(np.asarray(values, dtype=np.float32).reshape(shape), ctx.device)
        self.is_transformed = False

    def setType(self, grid_type):
        self.type = grid_type

    def getType(self):
        return self.type

    def getIsTransformed(self):
        return self.is_transformed

    def fftInPlace(self):
        assert not self.is_transformed
        self.ctx.fft_r2c(self.t, self.type)
        self.is_transformed = True

    def invFFTInPlace(self):
        assert self.is_transformed
        self.ctx.fft_c2r(self.t, self.type)
        self.is_transformed = False

    def numpy(self):
        return self.t.cpu().numpy()


class Crava:
    """The hot path of the reference's Crava on device grids.

    computePostMeanResidAndFFTCov: transformed means / stacks in, posterior
    mean (real domain), residual (transformed) and posterior covariance
    (transformed) out, as src/crava.cpp:887-1295 leaves them (the means are
    inverse transformed at :1181-1183; residuals and covariances stay in the
    Fourier domain)."""

    def __init__(self, ctx: Context, mu, data, cov, err_corr):
        self.ctx = ctx
        self.mu, self.data, self.cov, self.err = mu, data, cov, err_corr

    def computePostMeanResidAndFFTCov(self, precision=None):
        for g in self.cov + [self.err]:
            if not g.getIsTransformed():
                g.fftInPlace()
        self.ctx.posterior([g.t for g in self.mu], [g.t for g in self.data],
                           [g.t for g in self.cov], self.err.t, precision)
        for g in self.mu:
            g.invFFTInPlace()
        return 0

    def getPostAlpha(self):
        return self.mu[0]

    def getPostBeta(self):
        return self.mu[1]

    def getPostRho(self):
        return self.mu[2]

    def simulate(self, seed, n_sim, first_index=0):
        """n_sim realisations (list of [alpha, beta, rho] FFTGrids)."""
        ctx = self.ctx
        outs = [FFTGrid(ctx, grid_type=PARAMETER) for _ in range(3 * n_sim)]
        ctx.simulate([g.t for g in self.cov], [g.t for g in self.mu], seed, first_index,
                     [o.t for o in outs])
        return [outs[3 * r: 3 * r + 3] for r in range(n_sim)]
