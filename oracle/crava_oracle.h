/*
 * crava_oracle.h -- CPU oracle for the Fourier-domain AVO inversion hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product (crava_b200/, include/)
 * links, loads or calls this code.  It is the checker that the CUDA path is
 * compared against: tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline leg are its only users.
 *
 * Two implementations export this interface:
 *   orc_*  crava_oracle.c   -- a plain-C restatement of the reference's
 *                              algorithm (own FFT, own complex Cholesky).
 *   ref_*  ref_harness.cpp  -- the reference's own FFTW 2.1.2, lib_matr.c
 *                              and random.cpp compiled from its sources,
 *                              driven in the order crava.cpp drives them.
 * The restatement is pinned against the harness by tests/test_oracle_pin.py.
 *
 * Grid layout (both): one float buffer of rsize = 2*(nxp/2+1)*nyp*nzp
 * floats, real index i + rnxp*j + rnxp*nyp*k, complex (re,im) pair index
 * i + cnxp*j + cnxp*nyp*k after the in-place transform
 * (src/fftgrid.cpp:63-66, 1418-1431, 1698 of the reference).
 */
#ifndef CRAVA_ORACLE_H
#define CRAVA_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Identical layout to crava_gpu_params in include/crava_gpu.h. */
typedef struct crava_oracle_params {
  int nxp, nyp, nzp;          /* padded grid                                */
  int ntheta;                 /* number of angle stacks                     */
  int nz;                     /* unpadded layers (realFrequency numerator)  */
  int precision;              /* ignored by the oracle                      */
  double lz;                  /* simbox thickness (ms)                      */
  double min_rel_thick;       /* simbox min relative thickness             */
  float low_cut, high_cut;    /* frequency band (Hz)                        */
  float wnc;                  /* white-noise component                      */
  int thickness_mode;         /* 0 constant thickness, 1 non-constant         */
  const float  *wavelet;      /* [ntheta][nzp] time samples, FFT order      */
  const float  *wavelet_norm; /* [ntheta] or NULL (time-domain L2 norm)     */
  const float  *A;            /* [ntheta][3] reflection matrix              */
  const double *theta_cov;    /* [ntheta][ntheta] errThetaCov               */
  const double *var0;         /* [3][3] prior variance priorVar0            */
} crava_oracle_params;

/* Grid types: FFTGrid::gridTypes (src/fftgrid.h:172). */
enum { ORC_DATA = 1, ORC_PARAMETER = 2, ORC_COVARIANCE = 3 };

/* Per-kz tables of the solve (see orc_kz_tables).  Sizes are per kz:
 *   wd  [nzp][ntheta]  complex  D(k)*conj-wavelet, K = diag(wd)*A
 *   e1  [nzp][ntheta]  complex  errMult1
 *   e2  [nzp][ntheta]  complex  errMult2
 *   e3  [nzp][ntheta]  float    errMult3 (all 1 for constant thickness)
 *   inv [nzp]          int      invert_frequency
 */

/* ---- restatement (crava_oracle.c) ---- */
int orc_fft_r2c(float *grid, int nxp, int nyp, int nzp, int type);
int orc_fft_c2r(float *grid, int nxp, int nyp, int nzp, int type);
int orc_kz_tables(const crava_oracle_params *p, float *wd, float *e1, float *e2,
                  float *e3, int *inv);
int orc_posterior_fp32(const crava_oracle_params *p, float *const *mu,
                       float *const *data, float *const *cov,
                       const float *err_corr, long long *chol_fail);
int orc_posterior_fp32_t(const crava_oracle_params *p, const float *wd,
                         const float *e1, const float *e2, const float *e3,
                         const int *inv, float *const *mu, float *const *data,
                         float *const *cov, const float *err_corr,
                         long long *chol_fail);
int orc_posterior_fp64(const crava_oracle_params *p, const float *const *mu,
                       const float *const *data, const float *const *cov,
                       const float *err_corr, double *const *mu_out,
                       double *const *cov_out, double *const *res_out,
                       long long *chol_fail);
int orc_unit_fp32(const crava_oracle_params *p, float *const *mu,
                  float *const *data, float *const *cov, float *err_corr,
                  long long *chol_fail);
unsigned int orc_rng_fill_normal(unsigned int seed, double *out, long long n);
unsigned int orc_noise_fill(float *grid, int nxp, int nyp, int nzp,
                            unsigned int seed);
int orc_sim_filter(int nxp, int nyp, int nzp, const float *const *cov,
                   float *const *seed, long long *chol_fail);
int orc_sim_filter_fp64(int nxp, int nyp, int nzp, const float *const *cov,
                        float *const *seed, long long *chol_fail);
/* Crava::computeSyntSeismic + computeSeismicImpedance (constant thickness):
 * m[3] real padded grids, out[ntheta] real padded grids; nx, ny, nz the
 * unpadded sizes; wavelet [ntheta][nzp], A [ntheta][3]. */
/* computeCircCorrT + makeCircCorrTPosDef (circ_corr_t [nzp]). */
int orc_circ_corr_t(const float *prior_corr_t, int n, int low_int_cut, int nzp,
                    float *circ_corr_t);
/* fillInParamCorr times var0 (six grids) and fillInErrCorr (one grid);
 * corr_xy [nyp][nxp], var0 [3][3]. */
int orc_fill_prior_cov(int nxp, int nyp, int nzp, const float *corr_xy,
                       const float *circ_corr_t, float grad_i, float grad_j,
                       const double *var0, float *const *cov);
int orc_fill_err_corr(int nxp, int nyp, int nzp, const float *corr_xy,
                      float grad_i, float grad_j, float *err_corr);
/* Time-lapse state (State4D).  Spectra are interleaved float pairs of n
 * bins; state grids in State4D's orders (mu: vp, vs, rho; ss/dd: (0,0)
 * (0,1) (0,2) (1,1) (1,2) (2,2); sd: 3x3 row-major), the current state's
 * covariance in the posterior's order (00, 11, 22, 01, 02, 12). */
void orc_state4d_merge(long long n, const float *const *ms, const float *const *md,
                       const float *const *ss, const float *const *dd,
                       const float *const *sd, float *const *mu, float *const *cov);
long long orc_state4d_split(long long n, float *const *ms, float *const *md,
                            float *const *ss, float *const *dd, float *const *sd,
                            const float *const *mu, const float *const *cov);
void orc_state4d_evolve(long long n, float *const *ms, float *const *md,
                        float *const *ss, float *const *dd, float *const *sd,
                        const double *E, const double *cm, const double *cc,
                        const float *lambda, float zero_scale);
/* Crava::divideDataByScaleWavelet without interpolateSeismic: data
 * [ntheta] real padded grids (in place), cov_col [nzp] covAlpha(0,0,k),
 * rel_thick [nyp][nxp], shift / gain [ntheta][ny][nx] or NULL. */
int orc_divide_data(const crava_oracle_params *p, float *const *data, const float *cov_col,
                    const double *rel_thick, int nx, int ny, float dz, const float *shift,
                    const float *gain);
/* multiplyDataByScaleWaveletAndWriteToFile before the file write, on
 * time-domain residual grids (in place). */
int orc_multiply_data(const crava_oracle_params *p, float *const *data, const double *rel_thick,
                      int nx, int ny, float dz, const float *shift, const float *gain);
/* FFTGrid::interpolateSeismic + extrapolateSeismic on one real padded
 * data grid, in place. */
int orc_interpolate_seismic(float *grid, int nxp, int nyp, int nzp, int nx, int ny, int nz,
                            float energy_threshold, int *n_interpolated, int *n_zero);
int orc_fill_gen_exp_corr(int nxp, int nyp, int nzp, double rx, double ry, double rz,
                          float grad_i, float grad_j, float *out);
int orc_synt_seismic(int nxp, int nyp, int nzp, int nx, int ny, int nz, int ntheta,
                     const float *A, const float *wavelet, const float *const *m,
                     float *const *out);

/* ---- reference harness (ref_harness.cpp, built into oracle/_ref) ---- */
int ref_fft_r2c(float *grid, int nxp, int nyp, int nzp, int type);
int ref_fft_c2r(float *grid, int nxp, int nyp, int nzp, int type);
int ref_kz_tables(const crava_oracle_params *p, float *wd, float *e1, float *e2,
                  float *e3, int *inv);
int ref_posterior_fp32(const crava_oracle_params *p, float *const *mu,
                       float *const *data, float *const *cov,
                       const float *err_corr, long long *chol_fail);
int ref_posterior_fp32_t(const crava_oracle_params *p, const float *wd,
                         const float *e1, const float *e2, const float *e3,
                         const int *inv, float *const *mu, float *const *data,
                         float *const *cov, const float *err_corr,
                         long long *chol_fail);
int ref_unit_fp32(const crava_oracle_params *p, float *const *mu,
                  float *const *data, float *const *cov, float *err_corr,
                  long long *chol_fail);
unsigned int ref_rng_fill_normal(unsigned int seed, double *out, long long n);
unsigned int ref_noise_fill(float *grid, int nxp, int nyp, int nzp,
                            unsigned int seed);
int ref_sim_filter(int nxp, int nyp, int nzp, const float *const *cov,
                   float *const *seed, long long *chol_fail);
int ref_circ_corr_t(const float *prior_corr_t, int n, int low_int_cut, int nzp,
                    float *circ_corr_t);
int ref_synt_seismic(int nxp, int nyp, int nzp, int nx, int ny, int nz, int ntheta,
                     const float *A, const float *wavelet, const float *const *m,
                     float *const *out);
int ref_divide_data(const crava_oracle_params *p, float *const *data, const float *cov_col,
                    const double *rel_thick, int nx, int ny, float dz, const float *shift,
                    const float *gain);
int ref_multiply_data(const crava_oracle_params *p, float *const *data, const double *rel_thick,
                      int nx, int ny, float dz, const float *shift, const float *gain);
void ref_state4d_merge(long long n, const float *const *ms, const float *const *md,
                       const float *const *ss, const float *const *dd,
                       const float *const *sd, float *const *mu, float *const *cov);
long long ref_state4d_split(long long n, float *const *ms, float *const *md,
                            float *const *ss, float *const *dd, float *const *sd,
                            const float *const *mu, const float *const *cov);

#ifdef __cplusplus
}
#endif
#endif
