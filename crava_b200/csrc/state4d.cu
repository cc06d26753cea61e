// state4d.cu -- the time-lapse (4-D) state on the device.
//
// Replaces State4D::merge, mergeCov, split and evolve (src/state4d.cpp:
// 90-159, 161-249, 251-525, 527-730), FFTGrid::fillInGenExpCorr
// (src/fftgrid.cpp:1167-1210) and their composition in
// ModelGeneral::advanceTime (src/modelgeneral.cpp:4722-4736).
//
// Every step is one pass over Fourier-domain grids with one thread per
// complex bin (the bins are independent): HBM-bound elementwise work,
// coalesced float2 loads and stores of each grid.  merge and split follow
// the reference's float operations in its order (this file is compiled
// with -fmad=false; lib_matr's Cholesky and substitutions are restated in
// lib_matr_ref.cuh), so their grids equal the reference's bit for bit.
// evolve computes in double as the reference's FLENS matrices do (each
// product-sum as a chain of fused multiply-adds, as an FMA-capable BLAS
// forms it) and rounds to float once.
#include <math.h>

#include "context.cuh"
#include "lib_matr_ref.cuh"

using namespace crava;

namespace {

constexpr int kThreads = 256;
// split and evolve hold ~170 registers a thread: 128-thread blocks, three
// resident per SM, so that one block's loads overlap another's arithmetic
constexpr int kHeavyThreads = 128;
constexpr int kHeavyBlocks = 3;
constexpr float kMissing = -99999.0f;  // RMISSING, src/definitions.h:35

// State4D's upper-triangle order (p, q) of a 3x3 block and the position of
// the same entry in the crava_gpu_grids covariance order.
// (Functions, so that unrolled loops fold them to register indexes.)
__host__ __device__ constexpr int kP(int r) { return r < 3 ? 0 : (r < 5 ? 1 : 2); }
__host__ __device__ constexpr int kQ(int r) { return r < 3 ? r : (r < 5 ? r - 2 : 2); }
constexpr int kUnitPos[6] = {0, 3, 4, 1, 5, 2};

struct StateGrids {
  float2 *ms[3], *md[3], *ss[6], *dd[6], *sd[9];
};

struct CurGrids {
  float2 *mu[3];
  float2 *cov[6];  // State4D order (p, q) = (kP(r), kQ(r))
};

struct S4Args {
  StateGrids st;
  CurGrids cur;
  long long n;  // complex bins
  unsigned long long *shortcuts;
};

__device__ __forceinline__ float2 cj(float2 a) { return make_float2(a.x, -a.y); }

// ------------------------------------------------------------------ merge
__global__ void __launch_bounds__(kThreads) k_merge(const __grid_constant__ S4Args a) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= a.n) return;
  if (a.cur.mu[0]) {
#pragma unroll
    for (int l = 0; l < 3; ++l) {
      const float2 s = a.st.ms[l][idx], d = a.st.md[l][idx];
      a.cur.mu[l][idx] = make_float2(s.x + d.x, s.y + d.y);
    }
  }
#pragma unroll
  for (int r = 0; r < 6; ++r) {
    const int l = kP(r), m = kQ(r);
    const float2 f_lm = a.st.ss[r][idx];               // F[l][m]
    const float2 f_l3m3 = a.st.dd[r][idx];             // F[l+3][m+3]
    const float2 f_l3m = cj(a.st.sd[3 * m + l][idx]);  // F[l+3][m] = conj(F[m][l+3])
    const float2 f_lm3 = a.st.sd[3 * l + m][idx];      // F[l][m+3]
    float2 v;
    v.x = f_lm.x; v.x += f_l3m3.x; v.x += f_l3m.x; v.x += f_lm3.x;
    v.y = f_lm.y; v.y += f_l3m3.y; v.y += f_l3m.y; v.y += f_lm3.y;
    a.cur.cov[r][idx] = v;
  }
}

// ------------------------------------------------------------------ split
// One complex multiply-accumulate step of lib_matrProdCpx /
// lib_matrProdMatVecCpx: x += a b, each part as x + (p - q) / x + (p + q).
__device__ __forceinline__ void cmac(float2 &x, float2 a, float2 b) {
  x.x += a.x * b.x - a.y * b.y;
  x.y += a.y * b.x + a.x * b.y;
}

__global__ void __launch_bounds__(kHeavyThreads, kHeavyBlocks) k_split(const __grid_constant__ S4Args a) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= a.n) return;
  // sigmaFullPrior (Hermitian, from its upper triangle) and muFullPrior
  float2 F[6][6];
#pragma unroll
  for (int r = 0; r < 6; ++r) {
    F[kP(r)][kQ(r)] = a.st.ss[r][idx];
    F[kP(r) + 3][kQ(r) + 3] = a.st.dd[r][idx];
  }
#pragma unroll
  for (int l = 0; l < 3; ++l)
#pragma unroll
    for (int m = 0; m < 3; ++m) F[l][m + 3] = a.st.sd[3 * l + m][idx];
#pragma unroll
  for (int l = 0; l < 6; ++l)
#pragma unroll
    for (int m = l + 1; m < 6; ++m) F[m][l] = cj(F[l][m]);
  float2 muF[6];
#pragma unroll
  for (int l = 0; l < 3; ++l) { muF[l] = a.st.ms[l][idx]; muF[l + 3] = a.st.md[l][idx]; }
  // current posterior: lower triangle copied from the upper (as read)
  float2 muP[3], SP[3][3];
#pragma unroll
  for (int l = 0; l < 3; ++l) muP[l] = a.cur.mu[l][idx];
#pragma unroll
  for (int r = 0; r < 6; ++r) {
    const float2 v = a.cur.cov[r][idx];
    SP[kP(r)][kQ(r)] = v;
    SP[kQ(r)][kP(r)] = v;
  }
  // derived prior quantities
  float2 muC[3], FvC[6][3], SC[3][3];
#pragma unroll
  for (int l = 0; l < 3; ++l) muC[l] = make_float2(muF[l].x + muF[l + 3].x, muF[l].y + muF[l + 3].y);
#pragma unroll
  for (int l = 0; l < 6; ++l)
#pragma unroll
    for (int m = 0; m < 3; ++m)
      FvC[l][m] = make_float2(F[l][m].x + F[l][m + 3].x, F[l][m].y + F[l][m + 3].y);
#pragma unroll
  for (int l = 0; l < 3; ++l)
#pragma unroll
    for (int m = 0; m < 3; ++m)
      SC[l][m] = make_float2(FvC[l][m].x + FvC[l + 3][m].x, FvC[l][m].y + FvC[l + 3][m].y);
  float2 Lc[3][3], B[3][6];
#pragma unroll
  for (int l = 0; l < 3; ++l)
#pragma unroll
    for (int m = 0; m < 3; ++m) Lc[l][m] = SC[l][m];
#pragma unroll
  for (int l = 0; l < 6; ++l)
#pragma unroll
    for (int m = 0; m < 3; ++m) B[m][l] = cj(FvC[l][m]);  // adjoint(sigmaFullVsCurrentPrior)
  const bool ok = chol_ref<3>(Lc) == 0;
  if (ok) {
    axeqb_ref<3, 6>(Lc, B);  // B = inv(sigmaCurrentPrior) adjoint(FvC)
#pragma unroll
    for (int l = 0; l < 3; ++l)
#pragma unroll
      for (int m = 0; m < 3; ++m) { SP[l][m].x -= SC[l][m].x; SP[l][m].y -= SC[l][m].y; }
    float2 H[3][6];  // (Sigma_post - Sigma_cur) B
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 6; ++j) {
        float2 x = make_float2(0.0f, 0.0f);
#pragma unroll
        for (int k = 0; k < 3; ++k) cmac(x, SP[i][k], B[k][j]);
        H[i][j] = x;
      }
    // sigmaFullPosterior = adjoint(B) H + sigmaFullPrior, upper triangle
#pragma unroll
    for (int l = 0; l < 6; ++l)
#pragma unroll
      for (int m = l; m < 6; ++m) {
        float2 x = make_float2(0.0f, 0.0f);
#pragma unroll
        for (int k = 0; k < 3; ++k) cmac(x, cj(B[k][l]), H[k][m]);
        x.x += F[l][m].x;
        x.y += F[l][m].y;
        F[l][m] = x;
      }
#pragma unroll
    for (int l = 0; l < 3; ++l) { muP[l].x -= muC[l].x; muP[l].y -= muC[l].y; }
#pragma unroll
    for (int l = 0; l < 6; ++l) {
      float2 x = make_float2(0.0f, 0.0f);
#pragma unroll
      for (int k = 0; k < 3; ++k) cmac(x, cj(B[k][l]), muP[k]);
      x.x += muF[l].x;
      x.y += muF[l].y;
      muF[l] = x;
    }
  } else if (a.shortcuts) {
    atomicAdd(a.shortcuts, 1ull);
  }
#pragma unroll
  for (int r = 0; r < 6; ++r) {
    a.st.ss[r][idx] = F[kP(r)][kQ(r)];
    a.st.dd[r][idx] = F[kP(r) + 3][kQ(r) + 3];
  }
#pragma unroll
  for (int l = 0; l < 3; ++l)
#pragma unroll
    for (int m = 0; m < 3; ++m) a.st.sd[3 * l + m][idx] = F[l][m + 3];
#pragma unroll
  for (int l = 0; l < 3; ++l) { a.st.ms[l][idx] = muF[l]; a.st.md[l][idx] = muF[l + 3]; }
}

// ----------------------------------------------------------------- evolve
struct EvolveArgs {
  StateGrids st;
  const float2 *lambda;
  long long n;
  double E[36], cm[6], cc[36];
  float zero_scale;  // float(sqrt(double(nxp nyp nzp)))
};

__global__ void __launch_bounds__(kHeavyThreads, kHeavyBlocks) k_evolve(const __grid_constant__ EvolveArgs a) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= a.n) return;
  const double lam = (double)a.lambda[idx].x;
  const float sc = idx == 0 ? a.zero_scale : 0.0f;
  double mr[6], mi[6];
#pragma unroll
  for (int l = 0; l < 3; ++l) {
    const float2 s = a.st.ms[l][idx], d = a.st.md[l][idx];
    mr[l] = s.x; mi[l] = s.y; mr[l + 3] = d.x; mi[l + 3] = d.y;
  }
#pragma unroll
  for (int d = 0; d < 6; ++d) {
    double xr = 0.0, xi = 0.0;
#pragma unroll
    for (int e = 0; e < 6; ++e) { xr = __fma_rn(a.E[6 * d + e], mr[e], xr); xi = __fma_rn(a.E[6 * d + e], mi[e], xi); }
    xr = __fma_rn(a.cm[d], (double)sc, xr);
    float2 *g = d < 3 ? a.st.ms[d] : a.st.md[d - 3];
    g[idx] = make_float2((float)xr, (float)xi);
  }
  // the full 6x6 matrix; both parts mirrored unchanged, as the reference
  // fills it (held as float: the grids' own values, widened exactly on use)
  float Sr[6][6], Si[6][6];
#pragma unroll
  for (int r = 0; r < 6; ++r) {
    const int p = kP(r), q = kQ(r);
    const float2 s = a.st.ss[r][idx], d = a.st.dd[r][idx];
    Sr[p][q] = s.x; Si[p][q] = s.y; Sr[q][p] = s.x; Si[q][p] = s.y;
    Sr[p + 3][q + 3] = d.x; Si[p + 3][q + 3] = d.y;
    Sr[q + 3][p + 3] = d.x; Si[q + 3][p + 3] = d.y;
  }
#pragma unroll
  for (int l = 0; l < 3; ++l)
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      const float2 v = a.st.sd[3 * l + m][idx];
      Sr[l][m + 3] = v.x; Si[l][m + 3] = v.y; Sr[m + 3][l] = v.x; Si[m + 3][l] = v.y;
    }
  // row i of T = E S, then row i of S' = T E^T (+ C lambda for the real
  // part); only the upper triangle is stored
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    double tr[6], ti[6];
#pragma unroll
    for (int j = 0; j < 6; ++j) {
      double xr = 0.0, xi = 0.0;
#pragma unroll
      for (int k = 0; k < 6; ++k) {
        xr = __fma_rn(a.E[6 * i + k], (double)Sr[k][j], xr);
        xi = __fma_rn(a.E[6 * i + k], (double)Si[k][j], xi);
      }
      tr[j] = xr; ti[j] = xi;
    }
#pragma unroll
    for (int j = i; j < 6; ++j) {
      double xr = 0.0, xi = 0.0;
#pragma unroll
      for (int k = 0; k < 6; ++k) { xr = __fma_rn(tr[k], a.E[6 * j + k], xr); xi = __fma_rn(ti[k], a.E[6 * j + k], xi); }
      xr = __fma_rn(a.cc[6 * i + j], lam, xr);
      const float2 v = make_float2((float)xr, (float)xi);
      if (j < 3) a.st.ss[i == 0 ? j : (i == 1 ? j + 2 : 5)][idx] = v;
      else if (i < 3) a.st.sd[3 * i + j - 3][idx] = v;
      else a.st.dd[i == 3 ? j - 3 : (i == 4 ? j - 1 : 5)][idx] = v;
    }
  }
}

// --------------------------------------------------------- gen exp corr
struct GenExpArgs {
  float *out;
  double rx2, ry2, rz2;
  float grad_i, grad_j;
  int nxp, nyp, nzp, rnxp;
};

__device__ __forceinline__ int cyc(int i, int n) {
  int c = i - n;
  if (i < -c) c = i;
  return c;
}

__global__ void __launch_bounds__(kThreads) k_gen_exp_corr(const __grid_constant__ GenExpArgs a) {
  const long long n = (long long)a.rnxp * a.nyp * a.nzp;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n) return;
  const int i = (int)(idx % a.rnxp);
  const long long jk = idx / a.rnxp;
  const int j = (int)(jk % a.nyp), k = (int)(jk / a.nyp);
  float value = kMissing;
  if (i < a.nxp) {
    const int ci = cyc(i, a.nxp), cj = cyc(j, a.nyp);
    float subK = __fadd_rn(__fadd_rn((float)k, __fmul_rn((float)ci, a.grad_i)),
                           __fmul_rn((float)cj, a.grad_j));
    // cyclic fold into [-nzp/2, nzp/2); the host bounds |subK| so that a
    // few steps suffice
    const double half = a.nzp / 2.0;
    for (int it = 0; it < 64 && (double)subK < -half; ++it) subK = __fadd_rn(subK, (float)a.nzp);
    for (int it = 0; it < 64 && (double)subK >= half; ++it) subK = __fsub_rn(subK, (float)a.nzp);
    const double q = __dadd_rn(__dadd_rn(__ddiv_rn((double)(float)(ci * ci), a.rx2),
                                         __ddiv_rn((double)(cj * cj), a.ry2)),
                               __ddiv_rn((double)__fmul_rn(subK, subK), a.rz2));
    value = (float)exp(-3.0 * sqrt(q));
  }
  a.out[idx] = value;
}

bool mis8(const void *p) { return !p || (reinterpret_cast<uintptr_t>(p) & 7u) != 0; }

int state_grids(const crava_gpu_state4d *s, StateGrids *g) {
  if (!s) return CRAVA_GPU_ERR_ARG;
  for (int l = 0; l < 3; ++l) {
    if (mis8(s->mu_static[l]) || mis8(s->mu_dynamic[l])) return CRAVA_GPU_ERR_ARG;
    g->ms[l] = reinterpret_cast<float2 *>(s->mu_static[l]);
    g->md[l] = reinterpret_cast<float2 *>(s->mu_dynamic[l]);
  }
  for (int r = 0; r < 6; ++r) {
    if (mis8(s->cov_ss[r]) || mis8(s->cov_dd[r])) return CRAVA_GPU_ERR_ARG;
    g->ss[r] = reinterpret_cast<float2 *>(s->cov_ss[r]);
    g->dd[r] = reinterpret_cast<float2 *>(s->cov_dd[r]);
  }
  for (int r = 0; r < 9; ++r) {
    if (mis8(s->cov_sd[r])) return CRAVA_GPU_ERR_ARG;
    g->sd[r] = reinterpret_cast<float2 *>(s->cov_sd[r]);
  }
  return CRAVA_GPU_OK;
}

// The current state's grids, covariance reordered from the crava_gpu_grids
// order to State4D's.  mu may be NULL when allow_no_mu.
int cur_grids(const float *const *mu, const float *const *cov, bool allow_no_mu, CurGrids *g) {
  if (!cov) return CRAVA_GPU_ERR_ARG;
  if (mu) {
    for (int l = 0; l < 3; ++l) {
      if (mis8(mu[l])) return CRAVA_GPU_ERR_ARG;
      g->mu[l] = const_cast<float2 *>(reinterpret_cast<const float2 *>(mu[l]));
    }
  } else {
    if (!allow_no_mu) return CRAVA_GPU_ERR_ARG;
    for (int l = 0; l < 3; ++l) g->mu[l] = nullptr;
  }
  for (int r = 0; r < 6; ++r) {
    const float *p = cov[kUnitPos[r]];
    if (mis8(p)) return CRAVA_GPU_ERR_ARG;
    g->cov[r] = const_cast<float2 *>(reinterpret_cast<const float2 *>(p));
  }
  return CRAVA_GPU_OK;
}

unsigned grid_of(long long n, int threads = kThreads) { return (unsigned)((n + threads - 1) / threads); }

int split_async(crava_gpu_ctx *c, const crava_gpu_state4d *state, const float *const *mu,
                const float *const *cov) {
  S4Args a{};
  int rc;
  if ((rc = state_grids(state, &a.st)) || (rc = cur_grids(mu, cov, false, &a.cur))) return rc;
  a.n = c->g.csize;
  a.shortcuts = &c->counters->chol_fail;
  CRAVA_CUDA_TRY(cudaMemsetAsync(c->counters, 0, sizeof(DevCounters), c->stream));
  k_split<<<grid_of(a.n, kHeavyThreads), kHeavyThreads, 0, c->stream>>>(a);
  CRAVA_LAUNCH_CHECK();
  return CRAVA_GPU_OK;
}

int read_shortcuts(crava_gpu_ctx *c, long long *out) {
  if (!out) return CRAVA_GPU_OK;
  unsigned long long h = 0;
  CRAVA_CUDA_TRY(cudaMemcpyAsync(&h, &c->counters->chol_fail, sizeof h, cudaMemcpyDeviceToHost,
                                 c->stream));
  CRAVA_CUDA_TRY(cudaStreamSynchronize(c->stream));
  *out = (long long)h;
  return CRAVA_GPU_OK;
}

}  // namespace

extern "C" {

int crava_gpu_state4d_merge(crava_gpu_ctx *c, const crava_gpu_state4d *state, float *const mu[3],
                            float *const cov[6]) {
  if (!c) return CRAVA_GPU_ERR_ARG;
  S4Args a{};
  int rc;
  if ((rc = state_grids(state, &a.st)) || (rc = cur_grids(mu, cov, true, &a.cur))) return rc;
  DeviceGuard guard(c->device);
  a.n = c->g.csize;
  k_merge<<<grid_of(a.n), kThreads, 0, c->stream>>>(a);
  CRAVA_LAUNCH_CHECK();
  return CRAVA_GPU_OK;
}

int crava_gpu_state4d_split(crava_gpu_ctx *c, const crava_gpu_state4d *state,
                            const float *const mu[3], const float *const cov[6],
                            long long *shortcut_bins) {
  if (!c) return CRAVA_GPU_ERR_ARG;
  DeviceGuard guard(c->device);
  int rc;
  if ((rc = split_async(c, state, mu, cov))) return rc;
  return read_shortcuts(c, shortcut_bins);
}

int crava_gpu_fill_gen_exp_corr(crava_gpu_ctx *c, double rx, double ry, double rz, float grad_i,
                                float grad_j, float *grid) {
  if (!c || mis8(grid)) return CRAVA_GPU_ERR_ARG;
  if (!(rx > 0.0) || !(ry > 0.0) || !(rz > 0.0) || !isfinite(rx) || !isfinite(ry) || !isfinite(rz))
    return CRAVA_GPU_ERR_ARG;
  // |subK| stays below a few nzp, so the cyclic fold ends within its limit
  const double reach = fabs((double)grad_i) * c->g.nxp + fabs((double)grad_j) * c->g.nyp;
  if (!isfinite(grad_i) || !isfinite(grad_j) || reach > 16.0 * c->g.nzp) return CRAVA_GPU_ERR_ARG;
  DeviceGuard guard(c->device);
  GenExpArgs a{};
  a.out = grid;
  a.rx2 = rx * rx; a.ry2 = ry * ry; a.rz2 = rz * rz;
  a.grad_i = grad_i; a.grad_j = grad_j;
  a.nxp = c->g.nxp; a.nyp = c->g.nyp; a.nzp = c->g.nzp; a.rnxp = c->g.rnxp;
  k_gen_exp_corr<<<grid_of(c->g.rsize), kThreads, 0, c->stream>>>(a);
  CRAVA_LAUNCH_CHECK();
  return CRAVA_GPU_OK;
}

int crava_gpu_state4d_evolve(crava_gpu_ctx *c, const crava_gpu_state4d *state,
                             const double evolution[36], const double mean_correction[6],
                             const double cov_correction[36], const float *lambda) {
  if (!c || !evolution || !mean_correction || !cov_correction || mis8(lambda))
    return CRAVA_GPU_ERR_ARG;
  EvolveArgs a{};
  int rc;
  if ((rc = state_grids(state, &a.st))) return rc;
  DeviceGuard guard(c->device);
  a.lambda = reinterpret_cast<const float2 *>(lambda);
  a.n = c->g.csize;
  for (int t = 0; t < 36; ++t) { a.E[t] = evolution[t]; a.cc[t] = cov_correction[t]; }
  for (int t = 0; t < 6; ++t) a.cm[t] = mean_correction[t];
  a.zero_scale = (float)sqrt((double)((long long)c->g.nxp * c->g.nyp * c->g.nzp));
  k_evolve<<<grid_of(a.n, kHeavyThreads), kHeavyThreads, 0, c->stream>>>(a);
  CRAVA_LAUNCH_CHECK();
  return CRAVA_GPU_OK;
}

int crava_gpu_state4d_advance_time(crava_gpu_ctx *c, const crava_gpu_state4d *state,
                                   int time_step, int nx, int ny, const double evolution[36],
                                   const double mean_correction[6],
                                   const double cov_correction[36], float *const mu[3],
                                   float *const cov[6], float *lambda_work,
                                   long long *shortcut_bins) {
  if (!c || !mu || !cov || time_step < 0 || nx < 1 || ny < 1 || nx > c->g.nxp || ny > c->g.nyp)
    return CRAVA_GPU_ERR_ARG;
  if (mis8(lambda_work) || !evolution || !mean_correction || !cov_correction) return CRAVA_GPU_ERR_ARG;
  DeviceGuard guard(c->device);
  int rc;
  // split: the inverted current state into the static and dynamic parts
  if ((rc = split_async(c, state, mu, cov))) return rc;
  // evolve: the time increment's correlation, then the transition
  const double rz = time_step == 0 ? 50.0 : 5.0;
  if ((rc = crava_gpu_fill_gen_exp_corr(c, (double)(float)nx / 3.0, (double)(float)ny / 3.0, rz,
                                        0.0f, 0.0f, lambda_work)))
    return rc;
  if ((rc = pass_forward(c, lambda_work, lambda_work, CRAVA_GRID_COVARIANCE))) return rc;
  if ((rc = crava_gpu_state4d_evolve(c, state, evolution, mean_correction, cov_correction,
                                     lambda_work)))
    return rc;
  // merge: the next prior of the current state, back to the time domain
  if ((rc = crava_gpu_state4d_merge(c, state, mu, cov))) return rc;
  for (int l = 0; l < 3; ++l)
    if ((rc = pass_inverse(c, mu[l], CRAVA_GRID_PARAMETER))) return rc;
  for (int r = 0; r < 6; ++r)
    if ((rc = pass_inverse(c, cov[r], CRAVA_GRID_COVARIANCE))) return rc;
  return read_shortcuts(c, shortcut_bins);
}

}  // extern "C"
