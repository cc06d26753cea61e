// sim.cu -- posterior realisations: seeded complex noise and the per-bin
// Cholesky filter.  Compiled with -fmad=false so the FP32 filter rounds
// like the reference's (libs/lib/lib_matr.c:78-167, 453-470).
//
// Replaces Crava::simulate (src/crava.cpp:1415-1599) per realisation:
//   FFTGrid::fillInComplexNoise x3 (src/fftgrid.cpp:1213-1263),
//   per bin: rebuild the Hermitian posterior 3x3 from 6 spectra, Cholesky,
//   seed <- L seed, zero on failure (src/crava.cpp:1482-1521),
//   invFFTInPlace x3 and add of the posterior mean (:1537-1573).
// The reference draws the noise from one sequential LCG; here every bin's
// value is a pure function of (seed, stream, bin) through Philox-4x32-10
// (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1, 2,
// 3", SC 2011) and a Box-Muller transform, so realisations match the
// reference in distribution, not in value.
#include <math.h>

#include "sim.cuh"

namespace crava {

namespace {

constexpr int kThreads = 256;

// ---------------------------------------------------------------- Philox-4x32-10
struct U4 { uint32_t x, y, z, w; };

__device__ __forceinline__ U4 philox_round(U4 c, uint32_t k0, uint32_t k1) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  uint32_t hi0 = __umulhi(M0, c.x), lo0 = M0 * c.x;
  uint32_t hi1 = __umulhi(M1, c.z), lo1 = M1 * c.z;
  return U4{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
}

__device__ __forceinline__ U4 philox10(U4 c, uint32_t k0, uint32_t k1) {
  const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    c = philox_round(c, k0, k1);
    k0 += W0; k1 += W1;
  }
  return c;
}

// Two independent N(0,1) values for (seed, stream, counter), Box-Muller.
__device__ __forceinline__ float2 normal2(uint64_t seed, uint64_t stream, uint64_t ctr) {
  U4 c{(uint32_t)ctr, (uint32_t)(ctr >> 32), (uint32_t)stream, (uint32_t)(stream >> 32)};
  U4 r = philox10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
  // u1 in (0, 1], u2 in [0, 1)
  float u1 = ((float)(r.x >> 8) + 1.0f) * (1.0f / 16777216.0f);
  float u2 = (float)(r.y >> 8) * (1.0f / 16777216.0f);
  float rad = sqrtf(-2.0f * logf(u1));
  float s, co;
  sincospif(2.0f * u2, &s, &co);
  return make_float2(rad * co, rad * s);
}

// Where the noise of bin i comes from, under FFTGrid::fillInComplexNoise's
// rules (src/fftgrid.cpp:1221-1257, including the parity test on the
// linear index for the last x plane): each independent draw is made at the
// counter of the bin the reference draws it for; a mirrored bin re-draws
// its partner.  kind 0: an independent complex value, 1: a self-conjugate
// bin (real), 2: the conjugate of the partner's value.
struct NoiseSite {
  uint64_t ctr;
  int kind;
};

__device__ __forceinline__ NoiseSite noise_site(long long i, int cnxp, int nyp, int nzp) {
  const long long xs = i % cnxp;
  if (xs == 0 || (xs == cnxp - 1 && (i % 2) == 1)) {
    const long long jk = (i - xs) / cnxp;
    const long long j = jk % nyp, k = jk / nyp;
    const long long jc = j == 0 ? 0 : nyp - j, kc = k == 0 ? 0 : nzp - k;
    const long long jkc = jc + kc * nyp;
    if (jkc == jk) return NoiseSite{(uint64_t)i, 1};
    if (jkc > jk) return NoiseSite{(uint64_t)i, 0};
    return NoiseSite{(uint64_t)(jkc * cnxp + xs), 2};
  }
  return NoiseSite{(uint64_t)i, 0};
}

__device__ __forceinline__ float2 noise_value(NoiseSite site, uint64_t seed, uint64_t stream) {
  const float sd = 0.70710678118654752440f;  // float(1/sqrt(2.0))
  const float2 n = normal2(seed, stream, site.ctr);
  if (site.kind == 1) return make_float2(n.x, 0.0f);
  if (site.kind == 2) return make_float2(sd * n.x, -(sd * n.y));
  return make_float2(sd * n.x, sd * n.y);
}

// The value FFTGrid::fillInComplexNoise puts in bin i.
__device__ __forceinline__ float2 noise_bin(long long i, int cnxp, int nyp, int nzp,
                                            uint64_t seed, uint64_t stream) {
  return noise_value(noise_site(i, cnxp, nyp, nzp), seed, stream);
}

__global__ void __launch_bounds__(kThreads) k_noise(float2 *g, long long csize, int cnxp, int nyp,
                                                    int nzp, uint64_t seed, uint64_t stream) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < csize) g[i] = noise_bin(i, cnxp, nyp, nzp, seed, stream);
}

// lib_matrCholCpx on the 3x3 posterior covariance (reference operation order).
__device__ __forceinline__ int chol3_ref(float2 (*m)[3]) {
  float2 lr;
  float help;
  float factor = m[0][0].x;
  if (factor <= 0) return 1;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) { m[i][j].x = m[i][j].x / factor; m[i][j].y = m[i][j].y / factor; }
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    if ((double)m[i][i].x <= 1e-20) return 1;
#pragma unroll
    for (int j = 0; j < i; ++j) {
      lr.x = 0.0f; lr.y = 0.0f;
#pragma unroll
      for (int k = 0; k < j; ++k) {
        lr.x += (m[i][k].x * m[j][k].x) + (m[i][k].y * m[j][k].y);
        lr.y += -(m[i][k].x * m[j][k].y) + (m[i][k].y * m[j][k].x);
      }
      help = m[j][j].x * m[j][j].x + m[j][j].y * m[j][j].y;
      m[i][j].x = ((m[i][j].x - lr.x) * m[j][j].x + (m[i][j].y - lr.y) * m[j][j].y) / help;
      m[i][j].y = ((m[i][j].y - lr.y) * m[j][j].x - (m[i][j].x - lr.x) * m[j][j].y) / help;
    }
    lr.x = 0.0f;
#pragma unroll
    for (int k = 0; k < i; ++k) lr.x += (m[i][k].x * m[i][k].x) + (m[i][k].y * m[i][k].y);
    lr.x = m[i][i].x - lr.x;
    if ((double)lr.x <= 1e-20) return 1;
    m[i][i].x = sqrtf(lr.x);
    m[i][i].y = 0.0f;
  }
  const float sf = sqrtf(factor);
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j <= i; ++j) { m[i][j].x *= sf; m[i][j].y *= sf; }
  return 0;
}

// seed <- L seed (lib_matrProdCholVec), zero on failure.  Returns failure.
__device__ __forceinline__ bool filter_bin(const float2 *const *cov, long long i, float2 z[3]) {
  float2 P[3][3];
  P[0][0] = cov[0][i]; P[1][1] = cov[1][i]; P[2][2] = cov[2][i];
  P[0][1] = cov[3][i]; P[0][2] = cov[4][i]; P[1][2] = cov[5][i];
  P[1][0] = make_float2(P[0][1].x, -P[0][1].y);
  P[2][0] = make_float2(P[0][2].x, -P[0][2].y);
  P[2][1] = make_float2(P[1][2].x, -P[1][2].y);
  if (chol3_ref(P) == 0) {
    float2 o[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      o[a] = make_float2(0.0f, 0.0f);
#pragma unroll
      for (int b = 0; b < a + 1; ++b) {
        o[a].x += P[a][b].x * z[b].x - P[a][b].y * z[b].y;
        o[a].y += P[a][b].x * z[b].y + P[a][b].y * z[b].x;
      }
    }
    z[0] = o[0]; z[1] = o[1]; z[2] = o[2];
    return false;
  }
  z[0] = z[1] = z[2] = make_float2(0.0f, 0.0f);
  return true;
}

struct FilterArgs {
  const float2 *cov[6];
  float2 *seed[3];
  long long csize;
  DevCounters *counters;
};

__device__ __forceinline__ void count_fail(DevCounters *c, bool fail) {
  unsigned m = __activemask();
  unsigned b = __ballot_sync(m, fail);
  if (b && (threadIdx.x & 31) == __ffs(m) - 1) atomicAdd(&c->chol_fail, (unsigned long long)__popc(b));
}

__global__ void __launch_bounds__(kThreads) k_filter(FilterArgs a) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.csize) return;
  float2 z[3] = {a.seed[0][i], a.seed[1][i], a.seed[2][i]};
  bool f = filter_bin(a.cov, i, z);
#pragma unroll
  for (int q = 0; q < 3; ++q) a.seed[q][i] = z[q];
  if (a.counters) count_fail(a.counters, f);
}

struct NoiseFilterArgs {
  const float2 *cov[6];
  float2 *out[3];
  long long csize;
  int cnxp, nyp, nzp;
  uint64_t seed, stream0;  // parameter p uses stream stream0 + p
  DevCounters *counters;
};

__global__ void __launch_bounds__(kThreads) k_noise_filter(NoiseFilterArgs a) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.csize) return;
  float2 z[3];
#pragma unroll
  for (int q = 0; q < 3; ++q) z[q] = noise_bin(i, a.cnxp, a.nyp, a.nzp, a.seed, a.stream0 + q);
  bool f = filter_bin(a.cov, i, z);
#pragma unroll
  for (int q = 0; q < 3; ++q) a.out[q][i] = z[q];
  if (a.counters) count_fail(a.counters, f);
}

// Several realisations per pass: the posterior Cholesky factor of each bin
// is computed once and applied to the noise of every realisation
// (realisation r, parameter p uses stream stream0 + 3 r + p).
constexpr int kMaxSimBatch = 8;
struct NoiseFilterMultiArgs {
  const float2 *cov[6];
  float2 *out[3 * kMaxSimBatch];
  int nreal;
  long long csize;
  int cnxp, nyp, nzp;
  uint64_t seed, stream0;
  const unsigned long long *epoch;  // optional device counter: stream0 += epoch_mul * (*epoch)
  unsigned long long epoch_mul;
  DevCounters *counters;
};

__global__ void __launch_bounds__(kThreads) k_noise_filter_multi(const __grid_constant__ NoiseFilterMultiArgs a) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.csize) return;
  float2 P[3][3];
  P[0][0] = a.cov[0][i]; P[1][1] = a.cov[1][i]; P[2][2] = a.cov[2][i];
  P[0][1] = a.cov[3][i]; P[0][2] = a.cov[4][i]; P[1][2] = a.cov[5][i];
  P[1][0] = make_float2(P[0][1].x, -P[0][1].y);
  P[2][0] = make_float2(P[0][2].x, -P[0][2].y);
  P[2][1] = make_float2(P[1][2].x, -P[1][2].y);
  const bool ok = chol3_ref(P) == 0;
  const uint64_t stream0 = a.stream0 + (a.epoch ? a.epoch_mul * *a.epoch : 0ull);
  const NoiseSite site = noise_site(i, a.cnxp, a.nyp, a.nzp);  // once per bin
  for (int r = 0; r < a.nreal; ++r) {
    float2 z[3], o[3];
#pragma unroll
    for (int q = 0; q < 3; ++q) z[q] = noise_value(site, a.seed, stream0 + 3ull * r + q);
#pragma unroll
    for (int p = 0; p < 3; ++p) {
      o[p] = make_float2(0.0f, 0.0f);
      if (ok) {
#pragma unroll
        for (int b = 0; b < p + 1; ++b) {
          o[p].x += P[p][b].x * z[b].x - P[p][b].y * z[b].y;
          o[p].y += P[p][b].x * z[b].y + P[p][b].y * z[b].x;
        }
      }
    }
#pragma unroll
    for (int p = 0; p < 3; ++p) a.out[3 * r + p][i] = o[p];
  }
  if (a.counters) {
    unsigned m = __activemask();
    unsigned b = __ballot_sync(m, !ok);
    if (b && (threadIdx.x & 31) == __ffs(m) - 1)
      atomicAdd(&a.counters->chol_fail, (unsigned long long)__popc(b) * (unsigned long long)a.nreal);
  }
}

struct SimAllArgs {
  SimVintage v[kMaxSimVintages];
  long long first_block[kMaxSimVintages + 1];  // prefix of the vintages' 256-bin blocks
  int nv;
  const unsigned long long *epoch;
};

__global__ void __launch_bounds__(kThreads) k_noise_filter_vintages(const __grid_constant__ SimAllArgs a) {
  const long long nblocks = a.first_block[a.nv];
  const unsigned long long ep = a.epoch ? *a.epoch : 0ull;
  for (long long w = blockIdx.x; w < nblocks; w += gridDim.x) {
    int v = 0;
    while (v + 1 < a.nv && w >= a.first_block[v + 1]) ++v;
    const SimVintage &V = a.v[v];
    const long long i = (w - a.first_block[v]) * kThreads + threadIdx.x;
    if (i < V.csize) {
      float2 P[3][3];
      P[0][0] = V.cov[0][i]; P[1][1] = V.cov[1][i]; P[2][2] = V.cov[2][i];
      P[0][1] = V.cov[3][i]; P[0][2] = V.cov[4][i]; P[1][2] = V.cov[5][i];
      P[1][0] = make_float2(P[0][1].x, -P[0][1].y);
      P[2][0] = make_float2(P[0][2].x, -P[0][2].y);
      P[2][1] = make_float2(P[1][2].x, -P[1][2].y);
      const bool ok = chol3_ref(P) == 0;
      const uint64_t stream0 = V.stream0 + V.epoch_mul * ep;
      const NoiseSite site = noise_site(i, V.cnxp, V.nyp, V.nzp);  // once per bin
      for (int r = 0; r < V.nsim; ++r) {
        float2 z[3], o[3];
#pragma unroll
        for (int q = 0; q < 3; ++q) z[q] = noise_value(site, V.seed, stream0 + 3ull * r + q);
#pragma unroll
        for (int p = 0; p < 3; ++p) {
          o[p] = make_float2(0.0f, 0.0f);
          if (ok) {
#pragma unroll
            for (int b = 0; b < p + 1; ++b) {
              o[p].x += P[p][b].x * z[b].x - P[p][b].y * z[b].y;
              o[p].y += P[p][b].x * z[b].y + P[p][b].y * z[b].x;
            }
          }
        }
#pragma unroll
        for (int p = 0; p < 3; ++p) V.out[3 * r + p][i] = o[p];
      }
      if (V.counters) {
        const unsigned m = __activemask();
        const unsigned b = __ballot_sync(m, !ok);
        if (b && (threadIdx.x & 31) == __ffs(m) - 1)
          atomicAdd(&V.counters->chol_fail, (unsigned long long)__popc(b) * (unsigned long long)V.nsim);
      }
    }
  }
}

}  // namespace

int noise_filter_vintages(const SimVintage *v, int nv, const unsigned long long *epoch, cudaStream_t s) {
  if (nv < 1 || nv > kMaxSimVintages) return CRAVA_GPU_ERR_ARG;
  SimAllArgs a;
  a.nv = nv;
  a.epoch = epoch;
  a.first_block[0] = 0;
  for (int k = 0; k < nv; ++k) {
    if (v[k].nsim < 1 || !v[k].out) return CRAVA_GPU_ERR_ARG;
    a.v[k] = v[k];
    a.first_block[k + 1] = a.first_block[k] + (v[k].csize + kThreads - 1) / kThreads;
  }
  // persistent: the resident blocks of the device walk every vintage's blocks
  int dev = 0, sms = 0, per = 0;
  CRAVA_CUDA_TRY(cudaGetDevice(&dev));
  CRAVA_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  CRAVA_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_noise_filter_vintages, kThreads, 0));
  const long long resident = (long long)(per > 0 ? per : 1) * sms;
  const long long nb = a.first_block[nv];
  dim3 grd((unsigned)(nb < resident ? nb : resident));
  k_noise_filter_vintages<<<grd, kThreads, 0, s>>>(a);
  CRAVA_LAUNCH_CHECK();
  return CRAVA_GPU_OK;
}

int noise_filter_multi(const Geom &g, const float2 *const cov[6], float2 *const *out, int nreal,
                       uint64_t seed, uint64_t stream0, const unsigned long long *epoch,
                       unsigned long long epoch_mul, DevCounters *counters, cudaStream_t s) {
  if (nreal < 1 || nreal > kMaxSimBatch) return CRAVA_GPU_ERR_ARG;
  NoiseFilterMultiArgs a;
  for (int t = 0; t < 6; ++t) a.cov[t] = cov[t];
  for (int k = 0; k < 3 * nreal; ++k) a.out[k] = out[k];
  a.nreal = nreal;
  a.csize = g.csize;
  a.cnxp = g.cnxp; a.nyp = g.nyp; a.nzp = g.nzp;
  a.seed = seed; a.stream0 = stream0;
  a.epoch = epoch; a.epoch_mul = epoch_mul;
  a.counters = counters;
  dim3 grd((unsigned)((g.csize + kThreads - 1) / kThreads));
  k_noise_filter_multi<<<grd, kThreads, 0, s>>>(a);
  CRAVA_LAUNCH_CHECK();
  return CRAVA_GPU_OK;
}

int noise_fill(const Geom &g, float2 *grid, uint64_t seed, uint64_t stream, cudaStream_t s) {
  dim3 grd((unsigned)((g.csize + kThreads - 1) / kThreads));
  k_noise<<<grd, kThreads, 0, s>>>(grid, g.csize, g.cnxp, g.nyp, g.nzp, seed, stream);
  CRAVA_LAUNCH_CHECK();
  return CRAVA_GPU_OK;
}

int sim_filter(const Geom &g, const float2 *const cov[6], float2 *const seed[3],
               DevCounters *counters, cudaStream_t s) {
  FilterArgs a;
  for (int t = 0; t < 6; ++t) a.cov[t] = cov[t];
  for (int q = 0; q < 3; ++q) a.seed[q] = seed[q];
  a.csize = g.csize;
  a.counters = counters;
  dim3 grd((unsigned)((g.csize + kThreads - 1) / kThreads));
  k_filter<<<grd, kThreads, 0, s>>>(a);
  CRAVA_LAUNCH_CHECK();
  return CRAVA_GPU_OK;
}

int noise_filter(const Geom &g, const float2 *const cov[6], float2 *const out[3],
                 uint64_t seed, uint64_t stream0, DevCounters *counters, cudaStream_t s) {
  NoiseFilterArgs a;
  for (int t = 0; t < 6; ++t) a.cov[t] = cov[t];
  for (int q = 0; q < 3; ++q) a.out[q] = out[q];
  a.csize = g.csize;
  a.cnxp = g.cnxp; a.nyp = g.nyp; a.nzp = g.nzp;
  a.seed = seed; a.stream0 = stream0;
  a.counters = counters;
  dim3 grd((unsigned)((g.csize + kThreads - 1) / kThreads));
  k_noise_filter<<<grd, kThreads, 0, s>>>(a);
  CRAVA_LAUNCH_CHECK();
  return CRAVA_GPU_OK;
}

}  // namespace crava
