/*
 * crava_gpu.h -- C ABI of the B200 (sm_100a) Fourier-domain Bayesian AVO
 * inversion hot path.
 *
 * Every entry point replaces one piece of the reference's CPU path and keeps
 * its data layout and semantics.  Grids are device (HBM) buffers in the
 * reference's padded layout: one float buffer of rsize = rnxp*nyp*nzp floats,
 * rnxp = 2*(nxp/2+1), real index i + rnxp*j + rnxp*nyp*k; after a forward
 * transform the same bytes hold cnxp*nyp*nzp complex (re, im) pairs at index
 * i + cnxp*j + cnxp*nyp*k, cnxp = nxp/2+1 (reference src/fftgrid.cpp:37-67,
 * 1418-1431, 1698).  All calls are asynchronous on the context's stream and
 * return a status code; nothing calls exit().  Plain C types only.
 */
#ifndef CRAVA_GPU_H
#define CRAVA_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CRAVA_GPU_MAX_THETA 8

/* Status codes (the reference returns int and calls exit(1) on fatal
 * conditions, e.g. src/crava.cpp:381-387; here every failure is a code). */
enum crava_gpu_status {
  CRAVA_GPU_OK = 0,
  CRAVA_GPU_ERR_ARG = 1,     /* bad size, pointer, count or parameter     */
  CRAVA_GPU_ERR_ALLOC = 2,   /* device or pinned-host allocation failed   */
  CRAVA_GPU_ERR_CUDA = 3,    /* a CUDA call or kernel launch failed       */
  CRAVA_GPU_ERR_TIMEOUT = 4, /* a bounded device wait gave up             */
  CRAVA_GPU_ERR_STATE = 5,   /* call out of order (e.g. no stats pending) */
  CRAVA_GPU_ERR_NODEV = 6,   /* no usable CUDA device                     */
  CRAVA_GPU_ERR_TOO_LARGE = 7 /* sizes beyond the static scratch of
                                 crava_gpu_posterior_noalloc              */
};

/* Grid types: FFTGrid::gridTypes (src/fftgrid.h:172).  They select the
 * scaling of fftInPlace / invFFTInPlace (src/fftgrid.cpp:1817, 1848-1859):
 * DATA and PARAMETER are scaled by 1/sqrt(N) both ways, COVARIANCE is
 * unscaled forward and scaled by 1/N on the inverse. */
enum crava_grid_type {
  CRAVA_GRID_DATA = 1,
  CRAVA_GRID_PARAMETER = 2,
  CRAVA_GRID_COVARIANCE = 3
};

/* Arithmetic of the per-bin solve. */
enum crava_solve_precision {
  CRAVA_SOLVE_FP64 = 0,  /* plain form: covariances, Cholesky and posterior in FP64     */
  CRAVA_SOLVE_MIXED = 1, /* FP32 build + Cholesky, one FP64 refinement step on the
                            residual, FP64 Schur subtraction for the posterior cov   */
  CRAVA_SOLVE_FP32 = 2   /* FP32 throughout, the reference's own arithmetic          */
};

/* Inversion parameters (what Crava::Crava gathers from ModelSettings,
 * ModelAVODynamic and SeismicParametersHolder, src/crava.cpp:73-120).
 * Host pointers; copied at crava_gpu_create. */
typedef struct crava_gpu_params {
  int nxp, nyp, nzp;          /* padded grid (2,3,5,7-smooth, as the reference pads)   */
  int ntheta;                 /* angle stacks, 1..CRAVA_GPU_MAX_THETA                  */
  int nz;                     /* unpadded layers: realFrequency = nz*1000/(lz*nzp)*k   */
  int precision;              /* default crava_solve_precision                         */
  double lz;                  /* simbox thickness in ms (Simbox::getlz)                */
  double min_rel_thick;       /* Simbox::getMinRelThick                                */
  float low_cut, high_cut;    /* frequency band in Hz (lowCut_, highCut_)              */
  float wnc;                  /* white-noise component (wnc_)                          */
  int thickness_mode;         /* 0: constant thickness (Simbox::getIsConstantThick), K =
                                 diag(D conj W) A; 1: non-constant thickness, the data
                                 already divided by the local scale wavelet
                                 (src/crava.cpp:1059-1083): K = diag(D) A, errMult1 =
                                 1/|W|, errMult2 = D3/|E3|, errMult3 = robust 1/|W(k)| */
  const float *wavelet;       /* [ntheta][nzp] wavelet samples in FFT order (rAmp_)    */
  const float *wavelet_norm;  /* [ntheta] Wavelet::getNorm, or NULL = time-domain norm */
  const float *A;             /* [ntheta][3] reflection matrix (A_)                    */
  const double *theta_cov;    /* [ntheta][ntheta] errThetaCov_                         */
  const double *var0;         /* [3][3] priorVar0_                                     */
} crava_gpu_params;

/* Device grids of one posterior.  mu: meanAlpha_, meanBeta_, meanRho_;
 * data: seisData_[l]; cov: covAlpha, covBeta, covRho, crCovAlphaBeta,
 * crCovAlphaRho, crCovBetaRho (SeismicParametersHolder order); err_corr: errCorr_. */
typedef struct crava_gpu_grids {
  float *mu[3];
  float *data[CRAVA_GPU_MAX_THETA];
  float *cov[6];
  float *err_corr;
} crava_gpu_grids;

/* Statistics of the last solve or simulation (replaces the reference's
 * silent prior fallback counts and its timing report). */
typedef struct crava_gpu_stats {
  long long chol_fail_bins;   /* inverted bins whose Cholesky failed (prior kept)     */
  long long nonfinite_bins;   /* bins with a non-finite output                         */
  float ms_forward;           /* device time of the forward transforms                 */
  float ms_solve;             /* device time of the per-bin solve                      */
  float ms_inverse;           /* device time of the inverse transforms                 */
  float ms_total;             /* device time of the whole call                         */
  long long refined_bins;     /* mixed form: inverted bins that took the FP64 refinement */
  long long tile_wait_timeouts; /* TMA tile loads of the z pass not seen complete within
                                   the wait limit (device-wide since the library was
                                   loaded; 0 in a healthy run, else the outputs of
                                   that pass are incomplete) */
} crava_gpu_stats;

typedef struct crava_gpu_ctx crava_gpu_ctx;

/* Creates a context on `device` issuing work on `stream` (a cudaStream_t,
 * NULL = the legacy default stream).  Builds the per-kz operator tables on
 * the device from the wavelets (the set-up of computePostMeanResidAndFFTCov,
 * src/crava.cpp:952-1058).  Replaces: Crava::Crava's set-up, src/crava.cpp:49-120. */
int crava_gpu_create(const crava_gpu_params *params, int device, void *stream,
                     crava_gpu_ctx **out);
int crava_gpu_destroy(crava_gpu_ctx *ctx);
const char *crava_gpu_status_string(int status);

/* In-place 3-D real-to-complex transform with the FFTGrid scaling of
 * grid_type.  Replaces FFTGrid::fftInPlace, src/fftgrid.cpp:1803-1829. */
int crava_gpu_fft_r2c(crava_gpu_ctx *ctx, float *grid, int grid_type);

/* In-place 3-D complex-to-real transform.  Replaces
 * FFTGrid::invFFTInPlace, src/fftgrid.cpp:1831-1862. */
int crava_gpu_fft_c2r(crava_gpu_ctx *ctx, float *grid, int grid_type);

/* The halves of a 3-D transform, for a grid split over GPUs (z slabs for
 * the x and y passes, (kx, ky) column shards for the z pass):
 * crava_gpu_fft_xy runs the x then y passes (dir -1, forward) or the y then
 * x passes (dir +1, inverse) over every plane of a grid of the context's
 * geometry (a slab: the context's nzp planes of a grid of nzp_full), the
 * real <-> half-complex x transform scaled as fftInPlace / invFFTInPlace
 * scale the whole grid of grid_type; crava_gpu_fft_z runs the unscaled
 * complex z pass over every column.  On one GPU (nzp_full = nzp) they
 * equal crava_gpu_fft_r2c / _c2r bit for bit. */
int crava_gpu_fft_xy(crava_gpu_ctx *ctx, float *grid, int dir, int grid_type, int nzp_full);
int crava_gpu_fft_z(crava_gpu_ctx *ctx, float *grid, int dir);

/* Per-(kx,ky,kz) posterior solve on transformed grids, in place:
 * mu <- posterior mean, data <- residual, cov <- posterior covariance
 * (err_corr is read).  Replaces the loop of
 * Crava::computePostMeanResidAndFFTCov, src/crava.cpp:1042-1151. */
int crava_gpu_posterior(crava_gpu_ctx *ctx, const crava_gpu_grids *grids,
                        int precision);

/* The whole posterior unit on real-domain grids, in place: forward
 * transforms of 3 means, ntheta stacks, 6 covariances and the noise
 * correlation; the solve; inverse transforms of 3 posterior means,
 * ntheta residuals and 6 posterior covariances.  Replaces
 * src/crava.cpp:175-190 (transforms), 1003, 1012, 1042-1151, 1181-1206, 218. */
int crava_gpu_posterior_unit(crava_gpu_ctx *ctx, const crava_gpu_grids *grids,
                             int precision);

/* The same unit reading the real inputs from `in` and writing every output
 * (and the transformed noise correlation) to `out`; `in` is left unchanged.
 * in == out gives crava_gpu_posterior_unit.  The first transform pass of
 * each grid reads `in` and writes `out`, so the traffic is that of the
 * in-place call. */
int crava_gpu_posterior_unit_oop(crava_gpu_ctx *ctx, const crava_gpu_grids *in,
                                 const crava_gpu_grids *out, int precision);

/* The same unit on HOST buffers (layout as above): uploads, runs and
 * downloads, overlapping copies with the transforms.  Host buffers should
 * be page-locked (see crava_gpu_host_register) for full PCIe speed.
 * Synchronous: returns when the outputs are in host memory.  This is the
 * entry point a CPU-resident Crava (fftw_malloc'd FFTGrid buffers) calls. */
int crava_gpu_posterior_unit_host(crava_gpu_ctx *ctx,
                                  const crava_gpu_grids *host_grids,
                                  int precision);

/* The host-buffer unit, asynchronous and two deep: uploads `in`, runs the
 * unit and downloads its outputs into `out` (out == in: in place, as
 * crava_gpu_posterior_unit_host), returning once the work is enqueued.
 * Consecutive calls alternate between two device work sets, so one call's
 * downloads overlap the next call's uploads (PCIe is full duplex).  The
 * host grids of a call must stay untouched until crava_gpu_host_wait
 * returns, and the `out` grids of calls in flight must be distinct; pin
 * them (crava_gpu_host_register) for asynchronous copies.  No counterpart
 * in the reference. */
int crava_gpu_posterior_unit_host_async(crava_gpu_ctx *ctx, const crava_gpu_grids *in,
                                        const crava_gpu_grids *out, int precision);
/* Waits for every asynchronous host-buffer unit of the context. */
int crava_gpu_host_wait(crava_gpu_ctx *ctx);
int crava_gpu_host_register(void *ptr, uint64_t bytes);
int crava_gpu_host_unregister(void *ptr);

/* Complex N(0,1) noise spectrum with the Hermitian rules of
 * FFTGrid::fillInComplexNoise (src/fftgrid.cpp:1213-1263), drawn from a
 * counter-based generator (Philox-4x32-10): bin values are a pure function
 * of (seed, stream_id, bin), so realisations are reproducible and resumable.
 * Replaces FFTGrid::fillInComplexNoise with RandomGen. */
int crava_gpu_noise_fill(crava_gpu_ctx *ctx, float *grid, uint64_t seed,
                         uint64_t stream_id);

/* Per-bin filter of three noise spectra through the Cholesky factor of the
 * posterior covariance spectra (FP32, as the reference): seed <- L seed,
 * zero where the factorisation fails.  Replaces src/crava.cpp:1482-1521. */
int crava_gpu_sim_filter(crava_gpu_ctx *ctx, const float *const cov[6],
                         float *const seed[3]);

/* `count` posterior realisations: noise + filter (one fused pass), inverse
 * transform (PARAMETER scaling), plus the real-domain posterior mean.
 * Realisation r uses stream ids 3*(first_index+r)+{0,1,2}.  out[3*r+p]
 * receives parameter p of realisation r (real grids).  cov: transformed
 * posterior covariance grids; post_mean: real-domain posterior means.
 * Replaces Crava::simulate, src/crava.cpp:1415-1599 (per realisation:
 * fillInComplexNoise x3, filter, invFFTInPlace x3, add). */
int crava_gpu_simulate(crava_gpu_ctx *ctx, const float *const cov[6],
                       const float *const post_mean[3], uint64_t seed,
                       int first_index, int count, float *const *out);

/* Waits for the context's stream and returns the statistics of the last
 * posterior / simulation call. */
int crava_gpu_get_stats(crava_gpu_ctx *ctx, crava_gpu_stats *stats);

/* Copies the device-built per-kz tables to host memory (for checking):
 * wd/e1/e2 [nzp][ntheta] complex, e3 [nzp][ntheta], inv [nzp]. */
int crava_gpu_kz_tables(crava_gpu_ctx *ctx, float *wd, float *e1, float *e2,
                        float *e3, int *inv);

/* Replaces the per-kz tables with caller-supplied ones (same layout as
 * crava_gpu_kz_tables), e.g. spectra computed by the reference's own FFTW
 * (src/crava.cpp:952-976, 1024-1058).  Host pointers; synchronous.  The
 * number of inverted planes sets the solve's launch shape, so a batch
 * graph captured on this context before the call must be created again. */
int crava_gpu_set_kz_tables(crava_gpu_ctx *ctx, const float *wd, const float *e1,
                            const float *e2, const float *e3, const int *inv);

/* The unit calls use the three-pass transforms (x, y, z) and the separate
 * per-bin solve by default.  After set_fused(ctx, 1) they use the fused
 * kernels instead (xy-plane transforms with a thread block cluster, and one
 * kernel for the z transform, the per-bin solve and the inverse z
 * transform) when the grid fits them and the precision is FP64 or MIXED.
 * The fused unit does not write the noise-correlation output grid (its
 * transform is kept internally); the three-pass unit leaves it transformed.
 * fused_available reports whether a call with `precision` could take the
 * fused path. */
int crava_gpu_set_fused(crava_gpu_ctx *ctx, int enable);
int crava_gpu_fused_available(crava_gpu_ctx *ctx, int precision);

/* Per-kernel device time (profiling mode records a CUDA event pair around
 * every launch of this context; off by default).  bytes_per_launch is the
 * algorithmic traffic of one launch: 2 grids for a transform pass (read +
 * write), (19 + 2 ntheta) grids for the solve, 9 grids for the noise filter. */
typedef struct crava_gpu_kernel_profile {
  char name[32];
  long long launches;
  double total_ms;
  double bytes_per_launch;
} crava_gpu_kernel_profile;
int crava_gpu_set_profiling(crava_gpu_ctx *ctx, int enable);
/* Synchronises, returns the accumulated records (up to max) and resets them;
 * *count receives the number of kernel kinds seen. */
int crava_gpu_get_profile(crava_gpu_ctx *ctx, crava_gpu_kernel_profile *out,
                          int max, int *count);

/* The per-bin posterior solve of crava_gpu_posterior for callers that cannot
 * allocate device memory: those whose HBM is owned by their own arena (a
 * framework's caching allocator, a pool reserved up front), where a
 * cudaMalloc fails or breaks the owner's accounting, and loops that cannot
 * take the synchronisation an allocation may imply.  Needs no context and
 * allocates nothing: its scratch (staged wavelets, per-kz tables, counters)
 * is one static device array of about 0.5 MB, held by every GPU that loads
 * the library until exit.  Limits: nzp <= 4096 and nzp * ntheta <= 16384,
 * else CRAVA_GPU_ERR_TOO_LARGE.  params: host; grids: transformed device
 * grids, updated in place as by crava_gpu_posterior; stream: a cudaStream_t
 * (NULL = legacy default stream) on the current device.  stats may be NULL
 * (asynchronous); if given, the call waits for the stream and fills the
 * failure counts (no timings).  nxp <= 8192 and nyp <= 4096 as for
 * crava_gpu_create.  The first call on a device sets up the scratch address
 * for that device -- make it before any stream capture.  That address is
 * cached for the life of the process and is stale after cudaDeviceReset:
 * do not call this entry point on a device after resetting it.
 * Calls overlapping on the GPU share the scratch and race: serialise them.
 * This entry point has no counterpart in the reference. */
int crava_gpu_posterior_noalloc(const crava_gpu_params *params,
                                const crava_gpu_grids *grids, int precision,
                                void *stream, crava_gpu_stats *stats);

/* Launch shapes of a context.  cols_y_tile / cols_z_tile: the y and z
 * column transforms (-1 the built-in choice, 0 the out-of-place pass, 1 the
 * register-resident pass of lengths 64/128/256/512, 8 or 16 columns per CTA
 * in the in-place pass, 2 (z only) the register-resident pass fed by TMA
 * tile loads, where the grid has an even number of lines per z plane;
 * lengths without compiled column kernels ignore it; the built-in z choice
 * is 2 where the fused x + y pass is in use and the grid allows it);
 * fused: the fused unit kernels (1) or the three passes (0); ms: one unit's
 * measured time (autotune output only); lanes: more than 1 lets the
 * transforms of different grids overlap on that many streams; rows_x: the x
 * pass of an even nxp (-1 built-in, 0 in-place pass, 1 register-resident
 * pass where nxp / 2 is 64..512).  All these choices give the same values
 * bit for bit.  xy_fused: the x and y passes as one thread-block-cluster
 * kernel where the geometry has one (256x256 and 128x128 planes; -1
 * built-in = on where the geometry has it, 0 off, 1 on; alone it is
 * slower than the separate register-resident passes on B200, in the unit
 * beside the TMA-fed z pass faster); it factorises the y transform
 * differently, so it agrees with the separate passes to float rounding,
 * not bit for bit.  kappa_refine (mixed form only, >= 0): an inverted bin whose
 * FP32 factor has (max L_ii / min L_ii)^2 above it takes one FP64
 * refinement step (0 refines every bin).  solve_shape: the launch shape of
 * the FP64 and mixed solves (-1 built-in: the Woodbury kernel (shape 6)
 * for FP64 on a context, the register-factor kernel with four 128-thread
 * blocks per SM (shape 3) for mixed; 0-5 square-root shapes for both, 6-8
 * Woodbury shapes for FP64); every square-root shape gives the same values
 * bit for bit, the Woodbury shapes agree with them to FP64 rounding.  No counterpart in the reference (FFTW plans
 * are fixed there). */
typedef struct crava_gpu_tuning {
  int cols_y_tile;
  int cols_z_tile;
  int fused;
  float ms;
  int lanes;   /* streams the unit's independent transforms run on (1..4) */
  int rows_x;
  float kappa_refine;
  int xy_fused;
  int solve_shape;
} crava_gpu_tuning;
int crava_gpu_get_tuning(crava_gpu_ctx *ctx, crava_gpu_tuning *out);
int crava_gpu_set_tuning(crava_gpu_ctx *ctx, const crava_gpu_tuning *t);

/* Autotuner: times the out-of-place unit (crava_gpu_posterior_unit_oop, in
 * -> out) under every launch-shape candidate of this geometry, reps timed
 * runs after one warm-up each, keeps the fastest on the context and
 * returns it in best (may be NULL).  in and out must not share a grid (the
 * inputs are read again by every candidate); out is overwritten.
 * Synchronous.  No counterpart in the reference. */
int crava_gpu_autotune(crava_gpu_ctx *ctx, const crava_gpu_grids *in,
                       const crava_gpu_grids *out, int precision, int reps,
                       crava_gpu_tuning *best);

/* Batch: several vintages (one context each, grids of any size), each
 * inverted and sampled, replayed as one CUDA graph launch.  Per vintage and
 * run: the posterior unit from `in` into `out` in the reference's order --
 * forward transforms, per-bin solve, inverse transforms of the posterior
 * means and residuals (Crava::computePostMeanResidAndFFTCov,
 * src/crava.cpp:952-1220) -- then nsim realisations from the posterior
 * covariance spectra (Crava::simulate, src/crava.cpp:1415-1599), then the
 * inverse transforms of the six covariance grids.  Run e (0, 1, ...) draws
 * realisations first_index + e*nsim + r, r < nsim, each with the noise of
 * crava_gpu_simulate for that index, so replays give fresh, reproducible
 * realisations.  Vintages run on separate branches of the graph, joined
 * for the realisation filter of all vintages, which is one persistent
 * launch (at most 16 vintages with realisations). */
typedef struct crava_gpu_vintage {
  crava_gpu_ctx *ctx;
  crava_gpu_grids in;      /* real inputs (read, not written)            */
  crava_gpu_grids out;     /* outputs, layout of crava_gpu_posterior_unit */
  int precision;
  int nsim;                /* realisations per run (0: none)             */
  uint64_t seed;
  uint64_t first_index;
  float *const *sim_out;   /* 3 * nsim real grids: alpha, beta, rho of
                              realisation r at 3 r + 0, 1, 2            */
} crava_gpu_vintage;

typedef struct crava_gpu_batch crava_gpu_batch;
enum crava_gpu_batch_flags {
  CRAVA_BATCH_AUTOTUNE = 1, /* autotune each context before capture      */
  CRAVA_BATCH_NO_GRAPH = 2  /* enqueue the work on every run, no graph   */
};
/* Validates, (optionally) autotunes, runs the batch once uncaptured (this
 * allocates the contexts' workspaces) and captures it into a graph.  The
 * warm-up run does not count as a run.  stream: the cudaStream_t the
 * batch runs on (NULL: the batch creates one).  All contexts on one device,
 * profiling off.  A context's workspaces and counters are shared with its
 * other calls: make none while a run is in flight (after
 * crava_gpu_batch_sync they are free again).  Each vintage's `in` and `out`
 * grids must be distinct (the inputs are read again on every run). */
int crava_gpu_batch_create(const crava_gpu_vintage *vintages, int n, int flags,
                           void *stream, crava_gpu_batch **out);
/* One run of every vintage: one cudaGraphLaunch on the batch stream
 * (asynchronous). */
int crava_gpu_batch_run(crava_gpu_batch *b);
/* Waits for the batch stream. */
int crava_gpu_batch_sync(crava_gpu_batch *b);
int crava_gpu_batch_destroy(crava_gpu_batch *b);

/* Gaussian log marginal likelihood of the seismic spectra and its adjoint.
 * Per inverted bin the data spectra are CN(K mu, M) with
 * M = K S K^H + N, the matrices of crava_gpu_posterior (K = diag(w) A,
 * w_l(kz) = s_l D(kz) conj(W_l(kz)), D(kz) = exp(2 pi i kz/nzp) - 1, S the
 * prior covariance, N the noise covariance with angle l's variance v_l
 * replacing theta_cov[l][l] at fixed correlations).  Returns
 *   L = sum_k c_k (-log det M_k - r_k^H M_k^-1 r_k),  r = d - K mu,
 * c_k = 2 off the kx = 0 and Nyquist planes (the stored half spectrum
 * stands for the full one), and dL/ds_l, dL/dv_l and dL/dW_l(kz) for
 * kz = 0 .. nzp/2 (complex: dL/dRe + i dL/dIm, W(nzp-kz) = conj(W(kz))).
 * grids: transformed, as crava_gpu_posterior takes them; not modified.
 * wavelet_scale [ntheta] (NULL: 1), noise_var [ntheta] (NULL: theta_cov
 * diagonal), wavelet_spec [nzp/2+1][ntheta] (re, im) (NULL: the DFT of the
 * context's wavelets).  Outputs may be NULL except loglik; failed_bins:
 * inverted bins whose M did not factor (left out).  The noise colouring
 * tables (e1, e2, e3) stay fixed.  FP64; synchronous.  Recomputes M and
 * its factor per bin (nothing of a forward pass is stored).  Its device
 * buffers (a few hundred KB) are kept on the context after the first
 * call; crava_gpu_get_stats then reports the kernel's device time as
 * ms_solve and ms_total (ms_forward and ms_inverse 0).  No
 * counterpart in the reference (its wavelet and noise estimates are not
 * gradient-based). */
int crava_gpu_loglik_grad(crava_gpu_ctx *ctx, const crava_gpu_grids *grids,
                          const double *wavelet_scale, const double *noise_var,
                          const double *wavelet_spec, double *loglik, double *g_scale,
                          double *g_noise, double *g_spec, long long *failed_bins);

/* Synthetic seismic, Crava::computeSyntSeismic (src/crava.cpp:1666-1719)
 * with computeSeismicImpedance (:1632-1663), constant thickness: for each
 * angle l, out[l] (real padded grid) receives imp = sum_p A[l][p] m_p on
 * every cell; on the traces x < nx, y < ny the layers z >= nz are replaced
 * by the reference's linear taper between layers 0 and nz-1, and the trace
 * is differenced forward in z (cyclic) and multiplied in the Fourier
 * domain by conj(W_l(kz)), the unnormalised spectrum of wavelet l (the
 * reference's getCAmp(k, 1)), then transformed back (1/nzp).  alpha, beta,
 * rho: real padded grids, not modified; nx, ny: unpadded lateral sizes
 * (0: nxp, nyp); nz: the context's.  nz = nzp - 1 is rejected (the
 * reference's taper divides by nzp - nz - 1).  Asynchronous. */
int crava_gpu_synt_seismic(crava_gpu_ctx *ctx, const float *alpha, const float *beta,
                           const float *rho, int nx, int ny, float *const *out);

/* Synthetic seismic with each trace's local wavelet, the general form of
 * Crava::computeSyntSeismic (src/crava.cpp:1666-1719): as
 * crava_gpu_synt_seismic, but the simbox trace (x, y) is filtered with
 * conj(getCAmp(k, sf)) of seisWavelet_[l]->createLocalWavelet1D(x, y) --
 * the wavelet shifted by shift[l][y][x] ms (divided by dz) and scaled by
 * gain[l][y][x] (Wavelet1D::shiftAndScale, WELLMISSING = none) -- at
 * sf = rel_thick[y][x] (Simbox::getRelThick; getLocalStretch is 1 for a
 * 1-D wavelet).  rel_thick: host [nyp][nxp]; shift, gain: host
 * [ntheta][ny][nx] or NULL; dz: the simbox's dz (> 0).  Synchronous in the
 * host arrays' upload, then asynchronous. */
int crava_gpu_synt_seismic_local(crava_gpu_ctx *ctx, const float *alpha, const float *beta,
                                 const float *rho, int nx, int ny, const double *rel_thick,
                                 float dz, const float *shift, const float *gain,
                                 float *const *out);

/* Circular temporal prior correlation on nzp samples:
 * SeismicParametersHolder::computeCircCorrT + makeCircCorrTPosDef
 * (src/seismicparametersholder.cpp:430-499): prior_corr_t[0..n) mirrored
 * onto the cyclic axis, its spectrum replaced by its modulus and zeroed for
 * k <= low_int_cut, transformed back and normalised to 1 at lag 0.  Host
 * computation (double-precision transforms), no context, no GPU.  Returns
 * CRAVA_GPU_ERR_ARG where the reference aborts (value at lag 0 <= 1e-5). */
int crava_gpu_circ_corr_t(const float *prior_corr_t, int n, int low_int_cut, int nzp,
                          float *circ_corr_t);

/* The six prior covariance grids on the device:
 * SeismicParametersHolder::initializeCorrelations
 * (src/seismicparametersholder.cpp:196-221), i.e. FFTGrid::fillInParamCorr
 * (src/fftgrid.cpp:1118-1164) times float(var0[p][q]) for (p, q) = (0,0),
 * (1,1), (2,2), (0,1), (0,2), (1,2).  corr_xy: host [nyp][nxp] lateral
 * correlation (ModelGeneral::findCorrXYGrid, src/modelgeneral.cpp:
 * 4072-4110, index i + nxp j); circ_corr_t: host [nzp]
 * (crava_gpu_circ_corr_t); grad_i, grad_j: the correlation direction
 * gradients.  cov: six device grids, written in the real padded layout
 * (padding cells RMISSING * var0, as the reference leaves them).  Same
 * float operations as the reference: bit-identical grids.  Asynchronous
 * (the host arrays are copied before the call returns). */
int crava_gpu_fill_prior_cov(crava_gpu_ctx *ctx, const float *corr_xy, const float *circ_corr_t,
                             float grad_i, float grad_j, float *const cov[6]);

/* The noise correlation grid errCorr on the device: FFTGrid::fillInErrCorr
 * (src/fftgrid.cpp:1064-1116), corr_xy as above.  Bit-identical to the
 * reference's grid.  Asynchronous. */
int crava_gpu_fill_err_corr(crava_gpu_ctx *ctx, const float *corr_xy, float grad_i, float grad_j,
                            float *err_corr);

/* Crava::divideDataByScaleWavelet (src/crava.cpp:591-722) with
 * computeAdjustmentFactor (:725-817) for one-dimensional wavelets: every
 * padded trace (i, j) of each angle's data grid (real padded layout, in
 * place) is tapered below nz, transformed along z, multiplied in the band
 * (lowCut, highCut) by the adjustment factor of its local wavelet (the
 * context's wavelet stretched by rel_thick[j][i] = Simbox::getRelThick,
 * shifted and scaled by the local time shift and gain), zeroed outside it
 * and transformed back; the row padding is kept.  The closing
 * FFTGrid::interpolateSeismic of low-energy traces is not part of it.
 *   cov_alpha: device, the real-domain prior covAlpha grid (its (0,0,k)
 *              column gives the temporal correlation, as
 *              getPriorCorrTFiltered reads it);
 *   rel_thick: host [nyp][nxp] doubles;
 *   nx, ny:    unpadded lateral sizes (the traces' mirrored simbox index);
 *   dz:        the wavelet's sampling interval (Wavelet::getDz), ms;
 *   shift, gain: host [ntheta][ny][nx] local time shift (ms) and gain
 *              grids (Wavelet::getLocalTimeshift / getLocalGainFactor;
 *              -999 = missing), or NULL.
 * Asynchronous on the context's stream. */
int crava_gpu_divide_data_by_scale_wavelet(crava_gpu_ctx *ctx, float *const *data,
                                           const float *cov_alpha, const double *rel_thick,
                                           int nx, int ny, float dz, const float *shift,
                                           const float *gain);

/* Crava::multiplyDataByScaleWaveletAndWriteToFile (src/crava.cpp:819-885)
 * up to its file write: each residual stack (transformed, as the solve
 * leaves it) is transformed back to the time domain (DATA scaling) and
 * every simbox trace (i < nx, j < ny) multiplied along z by the conjugate
 * spectrum of its local wavelet stretched by rel_thick[j][i], shifted and
 * scaled by the local shift and gain (Wavelet::getCAmp(k, scale)); the
 * other traces keep their values.  rel_thick, dz, shift, gain as for
 * crava_gpu_divide_data_by_scale_wavelet (shift / gain indexed by the
 * trace itself).  Asynchronous. */
int crava_gpu_multiply_data_by_scale_wavelet(crava_gpu_ctx *ctx, float *const *resid,
                                             const double *rel_thick, int nx, int ny, float dz,
                                             const float *shift, const float *gain);

/* FFTGrid::interpolateSeismic (src/fftgrid.cpp:2564-2654) with
 * interpolateTrace and extrapolateSeismic (:2658-2731), the step that
 * closes divideDataByScaleWavelet (src/crava.cpp:690): traces of the nx x
 * ny simbox whose energy over the nz samples is at most energy_threshold
 * times the mean energy are replaced, in the reference's order, by the
 * mean of their good neighbours; then every padded trace outside the box
 * of good traces takes its fill trace times the cube of the taper.  grid:
 * one device data grid (real padded layout, in place).  n_interpolated,
 * n_zero (may be NULL): the traces found bad, and of those with zero
 * energy.  Synchronous (the trace flags are walked on the host). */
int crava_gpu_interpolate_seismic(crava_gpu_ctx *ctx, float *grid, int nx, int ny,
                                  float energy_threshold, int *n_interpolated, int *n_zero);

/* Simbox geometry stored in the header of a .crava grid file
 * (FFTGrid::writeCravaFile, src/fftgrid.cpp:2399-2433). */
typedef struct crava_gpu_grid_header {
  double x0, y0, dx, dy;
  int nx, ny;
  double il0, xl0, il_step_x, il_step_y, xl_step_x, xl_step_y, angle;
} crava_gpu_grid_header;

/* FFTGrid::writeCravaFile / readCravaFile (src/fftgrid.cpp:2399-2487) for a
 * device grid (real padded layout): the reference's big-endian binary
 * format, byte-swapped on the device, moved through a pinned staging buffer
 * of the context.  read rejects a file whose rnxp, nyp, nzp differ from the
 * context's (CRAVA_GPU_ERR_ARG, as the reference throws); header may be
 * NULL.  Synchronous. */
int crava_gpu_crava_file_write(crava_gpu_ctx *ctx, const char *path, const float *grid,
                               const crava_gpu_grid_header *header);
int crava_gpu_crava_file_read(crava_gpu_ctx *ctx, const char *path, float *grid,
                              crava_gpu_grid_header *header);

/* The time-lapse state of State4D (src/state4d.h:44-106): the static and
 * dynamic parts of the prior, as Fourier-domain device grids (padded real
 * layout holding the transformed spectra), in the reference's own orders.
 *   mu_static, mu_dynamic: vp, vs, rho;
 *   cov_ss, cov_dd: (vp,vp) (vp,vs) (vp,rho) (vs,vs) (vs,rho) (rho,rho) of
 *     the static-static and dynamic-dynamic blocks;
 *   cov_sd: static (vp,vs,rho) x dynamic (vp,vs,rho), row-major. */
typedef struct crava_gpu_state4d {
  float *mu_static[3];
  float *mu_dynamic[3];
  float *cov_ss[6];
  float *cov_dd[6];
  float *cov_sd[9];
} crava_gpu_state4d;

/* State4D::merge (src/state4d.cpp:90-159) and mergeCov (:161-249): the
 * current state's prior, mu = static + dynamic and cov = the sum of the
 * four blocks, written into Fourier-domain grids.  mu may be NULL
 * (mergeCov only).  cov in the crava_gpu_grids order (covAlpha, covBeta,
 * covRho, crCovAlphaBeta, crCovAlphaRho, crCovBetaRho).  The reference's
 * float additions in its order: bit-identical grids.  Asynchronous. */
int crava_gpu_state4d_merge(crava_gpu_ctx *ctx, const crava_gpu_state4d *state,
                            float *const mu[3], float *const cov[6]);

/* State4D::split (src/state4d.cpp:251-525): the inverted current state
 * (Fourier-domain posterior mu and cov, crava_gpu_grids order) spread back
 * over the static and dynamic parts, per bin
 *   B = Sigma_cur^-1 Sigma_cur,full (lib_matr Cholesky, 6 right-hand sides),
 *   Sigma_full += B^H (Sigma_post - Sigma_cur) B,  mu_full += B^H (mu_post - mu_cur);
 * bins whose 3x3 Cholesky fails keep the prior (counted in
 * crava_gpu_stats.chol_fail_bins, and in *shortcut_bins when that is not
 * NULL, which makes the call synchronous).  The reference's float
 * operations in its order: bit-identical grids.  Updates state in place. */
int crava_gpu_state4d_split(crava_gpu_ctx *ctx, const crava_gpu_state4d *state,
                            const float *const mu[3], const float *const cov[6],
                            long long *shortcut_bins);

/* FFTGrid::fillInGenExpCorr (src/fftgrid.cpp:1167-1210): the generalised
 * exponential correlation exp(-3 sqrt((i/rx)^2 + (j/ry)^2 + (k/rz)^2)) on
 * the cyclic padded grid, k counter-rotated by the gradients; real padded
 * layout, padding cells RMISSING.  Asynchronous. */
int crava_gpu_fill_gen_exp_corr(crava_gpu_ctx *ctx, double rx, double ry, double rz,
                                float grad_i, float grad_j, float *grid);

/* State4D::evolve (src/state4d.cpp:527-730): the forward transition of the
 * full state in time, per bin (double arithmetic, rounded to float once)
 *   mu' = E mu + c_mu s (s = sqrt(nxp nyp nzp) at the zero bin, else 0),
 *   Sigma' = E Sigma E^T + C Re(lambda)  (imaginary part: E Im(Sigma) E^T),
 * E the [6][6] row-major evolution matrix, c_mu [6] and C [6][6] row-major
 * the correction terms (TimeEvolution::getEvolutionMatrix,
 * getMeanCorrectionTerm, getCovarianceCorrectionTerm), lambda the
 * transformed correlation grid of the time increment (COVARIANCE
 * transform of crava_gpu_fill_gen_exp_corr).  Updates state in place.
 * Asynchronous. */
int crava_gpu_state4d_evolve(crava_gpu_ctx *ctx, const crava_gpu_state4d *state,
                             const double evolution[36], const double mean_correction[6],
                             const double cov_correction[36], const float *lambda);

/* ModelGeneral::advanceTime (src/modelgeneral.cpp:4722-4736): split the
 * inverted current state (Fourier-domain mu, cov) into the state, build
 * the time-increment correlation (fillInGenExpCorr(nx/3, ny/3, 50 at step 0
 * else 5), forward transformed into lambda_work), evolve, merge the next
 * prior back into mu and cov and transform those to the time domain
 * (PARAMETER for mu, COVARIANCE for cov).  nx, ny: the unpadded lateral
 * sizes.  shortcut_bins as in crava_gpu_state4d_split. */
int crava_gpu_state4d_advance_time(crava_gpu_ctx *ctx, const crava_gpu_state4d *state,
                                   int time_step, int nx, int ny, const double evolution[36],
                                   const double mean_correction[6],
                                   const double cov_correction[36], float *const mu[3],
                                   float *const cov[6], float *lambda_work,
                                   long long *shortcut_bins);

/* Number of kernels this library launched so far in this process. */
long long crava_gpu_launch_count(void);

#ifdef __cplusplus
}
#endif
#endif
