// prior.cu -- prior and noise covariance grids built on the device.
//
// Replaces, for the grids the posterior unit reads:
//   SeismicParametersHolder::initializeCorrelations
//     (src/seismicparametersholder.cpp:196-221): the six prior covariance
//     grids = FFTGrid::fillInParamCorr (src/fftgrid.cpp:1118-1164) times
//     Sigma0_pq (FFTGrid::multiplyByScalar, :1992-2000, padding included);
//   FFTGrid::fillInErrCorr (src/fftgrid.cpp:1064-1116): the lateral noise
//     correlation at the (gradient-shifted) first layer;
//   SeismicParametersHolder::computeCircCorrT + makeCircCorrTPosDef
//     (src/seismicparametersholder.cpp:430-499): the circular temporal
//     correlation (host code, one short 1-D transform).
// The fills are elementwise and follow the reference's float operations
// one by one (no fused multiply-add), so their grids equal the reference's
// bit for bit.  One thread writes one real cell of all six grids.
#include <math.h>

#include <vector>

#include "context.cuh"

using namespace crava;

namespace {

constexpr int kThreads = 256;
constexpr float kMissing = -99999.0f;  // RMISSING, src/definitions.h:35

struct FillArgs {
  const float *corr_xy;   // [nyp][nxp]
  const float *circ;      // [nzp]
  float *out[6];
  float scale[6];         // float(Sigma0_pq); 1 and one grid for the noise correlation
  int nout;
  float grad_i, grad_j;
  int nxp, nyp, nzp, rnxp;
};

// cycleI / cycleJ of the fill loops: the signed lateral offset of a cell.
__device__ __forceinline__ int cyc(int i, int n) {
  int c = i - n;
  if (i < -c) c = i;
  return c;
}

// subK = k + cycleI gradI + cycleJ gradJ in the reference's float order.
__device__ __forceinline__ float sub_k(int k, int ci, int cj, float gi, float gj) {
  return __fadd_rn(__fadd_rn((float)k, __fmul_rn((float)ci, gi)), __fmul_rn((float)cj, gj));
}

__global__ void __launch_bounds__(kThreads) k_fill_param(const __grid_constant__ FillArgs a) {
  const long long n = (long long)a.rnxp * a.nyp * a.nzp;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n) return;
  const int i = (int)(idx % a.rnxp);
  const long long jk = idx / a.rnxp;
  const int j = (int)(jk % a.nyp), k = (int)(jk / a.nyp);
  float value = kMissing;
  if (i < a.nxp) {
    float subK = sub_k(k, cyc(i, a.nxp), cyc(j, a.nyp), a.grad_i, a.grad_j);
    int baseK = (int)floorf(subK);
    subK = __fsub_rn(subK, (float)baseK);
    baseK %= a.nzp;
    if (baseK < 0) baseK += a.nzp;
    value = __fmul_rn(__fsub_rn(1.0f, subK), __ldg(a.circ + baseK));
    value = __fadd_rn(value, __fmul_rn(subK, __ldg(a.circ + (baseK != a.nzp - 1 ? baseK + 1 : 0))));
    value = __fmul_rn(value, __ldg(a.corr_xy + i + (long long)a.nxp * j));
  }
#pragma unroll
  for (int t = 0; t < 6; ++t)
    if (t < a.nout) a.out[t][idx] = __fmul_rn(value, a.scale[t]);
}

__global__ void __launch_bounds__(kThreads) k_fill_err(const __grid_constant__ FillArgs a) {
  const long long n = (long long)a.rnxp * a.nyp * a.nzp;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n) return;
  const int i = (int)(idx % a.rnxp);
  const long long jk = idx / a.rnxp;
  const int j = (int)(jk % a.nyp), k = (int)(jk / a.nyp);
  const int range = 1;
  float value = kMissing;
  if (i < a.nxp) {
    float subK = sub_k(k, cyc(i, a.nxp), cyc(j, a.nyp), a.grad_i, a.grad_j);
    if (fabsf(subK) < (float)range || fabsf(__fsub_rn(subK, (float)a.nzp)) < (float)range) {
      int baseK = (int)subK;
      subK = __fsub_rn(subK, (float)baseK);
      while (baseK < -range) baseK += a.nzp;
      while (baseK >= range) baseK -= a.nzp;
      if (baseK < 0) subK = __fsub_rn(1.0f, subK);
      value = __fmul_rn(__fsub_rn(1.0f, subK), __ldg(a.corr_xy + i + (long long)a.nxp * j));
    } else {
      value = 0.0f;
    }
  }
  a.out[0][idx] = value;
}

bool mis8(const void *p) { return !p || (reinterpret_cast<uintptr_t>(p) & 7u) != 0; }

// Device copies of the lateral and temporal correlations (context-owned).
int upload_corr(crava_gpu_ctx *c, const float *corr_xy, const float *circ) {
  const size_t nxy = (size_t)c->g.nxp * c->g.nyp, nz = (size_t)c->g.nzp;
  if (!c->prior_buf) {
    if (cudaMalloc(&c->prior_buf, (nxy + nz) * sizeof(float)) != cudaSuccess) {
      c->prior_buf = nullptr;
      return CRAVA_GPU_ERR_ALLOC;
    }
  }
  CRAVA_CUDA_TRY(cudaMemcpyAsync(c->prior_buf, corr_xy, nxy * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  if (circ)
    CRAVA_CUDA_TRY(cudaMemcpyAsync(c->prior_buf + nxy, circ, nz * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  return CRAVA_GPU_OK;
}

}  // namespace

extern "C" {

int crava_gpu_circ_corr_t(const float *prior_corr_t, int n, int low_int_cut, int nzp,
                          float *circ_corr_t) {
  if (!prior_corr_t || !circ_corr_t || n < 1 || nzp < 2 || prior_corr_t[0] == 0.0f)
    return CRAVA_GPU_ERR_ARG;
  // computeCircCorrT: mirror the correlation onto the cyclic axis
  std::vector<double> c(nzp);
  for (int k = 0; k < nzp; ++k) {
    const int refk = k < nzp / 2 + 1 ? k : nzp - k;
    c[k] = refk < n ? (double)prior_corr_t[refk] : 0.0;
  }
  // makeCircCorrTPosDef: |spectrum|, zero up to low_int_cut, back (the
  // unnormalised pair of transforms), normalised by the value at lag 0
  const int cn = nzp / 2 + 1;
  std::vector<double> mag(cn);
  for (int k = 0; k < cn; ++k) {
    double re = 0.0, im = 0.0;
    for (int t = 0; t < nzp; ++t) {
      const double ang = -2.0 * M_PI * (double)(((long long)k * t) % nzp) / nzp;
      re += c[t] * cos(ang);
      im += c[t] * sin(ang);
    }
    mag[k] = k <= low_int_cut ? 0.0 : (double)(float)sqrt(re * re + im * im);
  }
  std::vector<double> back(nzp);
  for (int t = 0; t < nzp; ++t) {
    double s = mag[0];
    for (int k = 1; k < cn; ++k) {
      const double w = (2 * k == nzp) ? 1.0 : 2.0;  // conjugate partner
      s += w * mag[k] * cos(2.0 * M_PI * (double)(((long long)k * t) % nzp) / nzp);
    }
    back[t] = s;
  }
  if (!((float)back[0] > 1.e-5f)) return CRAVA_GPU_ERR_ARG;  // the reference aborts here
  const float scale = 1.0f / (float)back[0];
  for (int t = 0; t < nzp; ++t) circ_corr_t[t] = (float)back[t] * scale;
  return CRAVA_GPU_OK;
}

int crava_gpu_fill_prior_cov(crava_gpu_ctx *c, const float *corr_xy, const float *circ_corr_t,
                             float grad_i, float grad_j, float *const cov[6]) {
  if (!c || !corr_xy || !circ_corr_t || !cov) return CRAVA_GPU_ERR_ARG;
  for (int t = 0; t < 6; ++t) if (mis8(cov[t])) return CRAVA_GPU_ERR_ARG;
  DeviceGuard guard(c->device);
  int rc;
  if ((rc = upload_corr(c, corr_xy, circ_corr_t))) return rc;
  FillArgs a{};
  a.corr_xy = c->prior_buf;
  a.circ = c->prior_buf + (size_t)c->g.nxp * c->g.nyp;
  const int pq[6][2] = {{0, 0}, {1, 1}, {2, 2}, {0, 1}, {0, 2}, {1, 2}};
  for (int t = 0; t < 6; ++t) {
    a.out[t] = cov[t];
    a.scale[t] = (float)c->var0[3 * pq[t][0] + pq[t][1]];
  }
  a.nout = 6;
  a.grad_i = grad_i; a.grad_j = grad_j;
  a.nxp = c->g.nxp; a.nyp = c->g.nyp; a.nzp = c->g.nzp; a.rnxp = c->g.rnxp;
  const long long n = c->g.rsize;
  k_fill_param<<<(unsigned)((n + kThreads - 1) / kThreads), kThreads, 0, c->stream>>>(a);
  CRAVA_LAUNCH_CHECK();
  return CRAVA_GPU_OK;
}

int crava_gpu_fill_err_corr(crava_gpu_ctx *c, const float *corr_xy, float grad_i, float grad_j,
                            float *err_corr) {
  if (!c || !corr_xy || mis8(err_corr)) return CRAVA_GPU_ERR_ARG;
  DeviceGuard guard(c->device);
  int rc;
  if ((rc = upload_corr(c, corr_xy, nullptr))) return rc;
  FillArgs a{};
  a.corr_xy = c->prior_buf;
  a.out[0] = err_corr;
  a.nout = 1;
  a.grad_i = grad_i; a.grad_j = grad_j;
  a.nxp = c->g.nxp; a.nyp = c->g.nyp; a.nzp = c->g.nzp; a.rnxp = c->g.rnxp;
  const long long n = c->g.rsize;
  k_fill_err<<<(unsigned)((n + kThreads - 1) / kThreads), kThreads, 0, c->stream>>>(a);
  CRAVA_LAUNCH_CHECK();
  return CRAVA_GPU_OK;
}

}  // extern "C"
