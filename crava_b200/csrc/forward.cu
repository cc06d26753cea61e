// forward.cu -- synthetic seismic (forward modelling) on the device.
//
// Replaces Crava::computeSyntSeismic (src/crava.cpp:1666-1719) with
// Crava::computeSeismicImpedance (:1632-1663), constant thickness (relative
// thickness and local stretch 1, no local shift or gain).  For angle l:
//   imp = A_l0 alpha + A_l1 beta + A_l2 rho           (every real cell)
//   per trace x < nx, y < ny: imp[z] for z >= nz replaced by the linear
//   taper fac ((z - nz) imp[0] + (nzp - z - 1) imp[nz - 1]),
//   fac = 1 / (nzp - nz - 1); then the cyclic forward difference, the
//   unnormalised FFT, multiplication by conj(W_l(kz)) and the inverse FFT
//   scaled by 1/nzp.
// The difference and the wavelet are applied as one spectral factor
//   H_l(kz) = (exp(2 pi i kz / nzp) - 1) conj(W_l(kz)) / nzp,
// Hermitian in kz (both factors are spectra of real sequences), so two
// adjacent real traces x = 2p, 2p + 1 are filtered together as one complex
// line a + i b: the real grid viewed as complex pairs is exactly the
// complex layout the z column transforms work on.  Traces outside
// x < nx, y < ny keep imp, as in the reference.
#include <math.h>

#include <vector>

#include "context.cuh"

using namespace crava;

namespace {

constexpr int kThreads = 256;

struct SyntArgs {
  const float2 *m[3];     // alpha, beta, rho as float2 pairs
  float2 *out;            // one angle's output grid as float2 pairs
  const float2 *H;        // [nzp] filter of this angle
  const float2 *tw;       // [nzp] e^{-2 pi i k / nzp}
  float A[3];
  int cnxp, nyp, nzp, nx, ny, nz;
};

// ((0 + alpha A0) + beta A1) + rho A2 with separate roundings, the
// reference's float sequence (no fused multiply-add), so the traces the
// reference leaves unfiltered match it bit for bit.
__device__ __forceinline__ float imp1(float x, float y, float z, const float *A) {
  float r = __fadd_rn(0.0f, __fmul_rn(x, A[0]));
  r = __fadd_rn(r, __fmul_rn(y, A[1]));
  return __fadd_rn(r, __fmul_rn(z, A[2]));
}

__device__ __forceinline__ float2 imp_at(const SyntArgs &a, long long idx) {
  const float2 x = a.m[0][idx], y = a.m[1][idx], z = a.m[2][idx];
  return make_float2(imp1(x.x, y.x, z.x, a.A), imp1(x.y, y.y, z.y, a.A));
}

__device__ __forceinline__ float taper(float v0, float vl, int z, int nz, int nzp) {
  const float fac = 1.0f / (float)(nzp - nz - 1);
  return fac * ((float)(z - nz) * v0 + (float)(nzp - z - 1) * vl);
}

// One CTA: TX complex lines (x pairs x0 .. x0 + TX - 1) at one y, all z.
template <int N, int TX>
__global__ void __launch_bounds__(kThreads) k_synt(const __grid_constant__ SyntArgs a) {
  extern __shared__ float2 sm[];
  float2 *twl = sm;
  float2 *buf = twl + N;
  const int x0 = blockIdx.x * TX, y = blockIdx.y;
  const int tid = threadIdx.x;
  const long long plane = (long long)a.cnxp * a.nyp;
  const long long base = x0 + (long long)a.cnxp * y;
  for (int i = tid; i < N; i += kThreads) twl[i] = a.tw[i];
  constexpr int ES = cols_pitch(TX);
  constexpr int PADR = cols_padr(N, TX);
  for (int idx = tid; idx < TX * N; idx += kThreads) {
    const int t = idx % TX, m = idx / TX;
    buf[pad_row<PADR>(m) * ES + t] = x0 + t < a.cnxp ? imp_at(a, base + m * plane + t) : make_float2(0.f, 0.f);
  }
  __syncthreads();
  if (y < a.ny && a.nz < N) {
    for (int idx = tid; idx < TX * (N - a.nz); idx += kThreads) {
      const int t = idx % TX, m = a.nz + idx / TX;
      const float2 v0 = buf[t], vl = buf[pad_row<PADR>(a.nz - 1) * ES + t];
      buf[pad_row<PADR>(m) * ES + t] = make_float2(taper(v0.x, vl.x, m, a.nz, N), taper(v0.y, vl.y, m, a.nz, N));
    }
  }
  __syncthreads();
  stockham_ip<N, -1, TX, 1, ES, kThreads, PADR>(buf, twl);
  __syncthreads();
  for (int idx = tid; idx < TX * N; idx += kThreads) {
    const int t = idx % TX, m = idx / TX;
    float2 *b = buf + pad_row<PADR>(m) * ES + t;
    *b = cmul(*b, __ldg(a.H + m));
  }
  __syncthreads();
  stockham_ip<N, 1, TX, 1, ES, kThreads, PADR>(buf, twl);
  __syncthreads();
  for (int idx = tid; idx < TX * N; idx += kThreads) {
    const int t = idx % TX, m = idx / TX;
    const int p = x0 + t;
    if (p >= a.cnxp) continue;
    const long long g = base + m * plane + t;
    float2 v = buf[pad_row<PADR>(m) * ES + t];
    const bool fx = 2 * p < a.nx, fy = 2 * p + 1 < a.nx;
    if (y >= a.ny || !fx || !fy) {
      const float2 raw = imp_at(a, g);
      if (y >= a.ny || !fx) v.x = raw.x;
      if (y >= a.ny || !fy) v.y = raw.y;
    }
    a.out[g] = v;
  }
}

// All angles in one pass: a CTA holds its TX lines of the three parameter
// grids in registers (read from HBM once) and, per angle, forms the
// impedance in shared memory, tapers, transforms, filters, transforms back
// and stores: 3 grid reads + nt writes instead of nt (3 reads + 1 write).
struct SyntAllArgs {
  const float2 *m[3];
  float2 *out[CRAVA_GPU_MAX_THETA];
  const float2 *H;  // [nt][nzp]
  const float2 *tw;
  float A[CRAVA_GPU_MAX_THETA][3];
  int nt, cnxp, nyp, nzp, nx, ny, nz;
};

template <int N, int TX>
__global__ void __launch_bounds__(kThreads, N == 256 ? 1 : 2) k_synt_all(const __grid_constant__ SyntAllArgs a) {
  static_assert((TX * N) % kThreads == 0, "whole elements per thread");
  constexpr int E = TX * N / kThreads;
  extern __shared__ float2 sm[];
  float2 *twl = sm;
  float2 *buf = twl + N;
  const int x0 = blockIdx.x * TX, y = blockIdx.y, tid = threadIdx.x;
  const long long plane = (long long)a.cnxp * a.nyp;
  const long long base = x0 + (long long)a.cnxp * y;
  for (int i = tid; i < N; i += kThreads) twl[i] = a.tw[i];
  float2 pm[3][E];
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const int idx = tid + e * kThreads, t = idx % TX, m = idx / TX;
    const bool in = x0 + t < a.cnxp;
#pragma unroll
    for (int q = 0; q < 3; ++q) pm[q][e] = in ? a.m[q][base + m * plane + t] : make_float2(0.f, 0.f);
  }
  for (int l = 0; l < a.nt; ++l) {
    const float A[3] = {a.A[l][0], a.A[l][1], a.A[l][2]};
    __syncthreads();  // the previous angle's stores have read buf
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int idx = tid + e * kThreads, t = idx % TX, m = idx / TX;
      buf[m * TX + t] = make_float2(imp1(pm[0][e].x, pm[1][e].x, pm[2][e].x, A),
                                    imp1(pm[0][e].y, pm[1][e].y, pm[2][e].y, A));
    }
    __syncthreads();
    if (y < a.ny && a.nz < N) {
      for (int idx = tid; idx < TX * (N - a.nz); idx += kThreads) {
        const int t = idx % TX, m = a.nz + idx / TX;
        const float2 v0 = buf[t], vl = buf[(a.nz - 1) * TX + t];
        buf[m * TX + t] = make_float2(taper(v0.x, vl.x, m, a.nz, N), taper(v0.y, vl.y, m, a.nz, N));
      }
    }
    __syncthreads();
    stockham_ip<N, -1, TX, 1, TX, kThreads>(buf, twl);
    const float2 *H = a.H + (long long)l * N;
    for (int idx = tid; idx < TX * N; idx += kThreads) {
      float2 *b = buf + idx;  // (m, t) at m TX + t = idx
      *b = cmul(*b, __ldg(H + idx / TX));
    }
    __syncthreads();
    stockham_ip<N, 1, TX, 1, TX, kThreads>(buf, twl);
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int idx = tid + e * kThreads, t = idx % TX, m = idx / TX;
      const int p = x0 + t;
      if (p >= a.cnxp) continue;
      float2 v = buf[m * TX + t];
      const bool fx = 2 * p < a.nx, fy = 2 * p + 1 < a.nx;
      if (y >= a.ny || !fx) v.x = imp1(pm[0][e].x, pm[1][e].x, pm[2][e].x, A);
      if (y >= a.ny || !fy) v.y = imp1(pm[0][e].y, pm[1][e].y, pm[2][e].y, A);
      a.out[l][base + m * plane + t] = v;
    }
  }
}

template <int N>
int launch_synt_all(const SyntAllArgs &a, cudaStream_t s) {
  constexpr int TX = 4;
  const size_t smem = sizeof(float2) * (N + (size_t)TX * N);
  int rc = func_smem((const void *)k_synt_all<N, TX>, smem);
  if (rc) return rc;
  const dim3 grd((unsigned)((a.cnxp + TX - 1) / TX), (unsigned)a.nyp);
  k_synt_all<N, TX><<<grd, kThreads, smem, s>>>(a);
  CRAVA_LAUNCH_CHECK();
  return CRAVA_GPU_OK;
}

// Generic lengths, step 1: impedance and taper written to the output grid.
__global__ void __launch_bounds__(kThreads) k_synt_imp(const __grid_constant__ SyntArgs a) {
  const long long plane = (long long)a.cnxp * a.nyp;
  const long long n = plane * a.nzp;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n) return;
  const int m = (int)(idx / plane);
  const long long col = idx - (long long)m * plane;
  const int y = (int)(col / a.cnxp);
  float2 v = imp_at(a, idx);
  if (y < a.ny && m >= a.nz) {
    const float2 v0 = imp_at(a, col), vl = imp_at(a, col + (long long)(a.nz - 1) * plane);
    v = make_float2(taper(v0.x, vl.x, m, a.nz, a.nzp), taper(v0.y, vl.y, m, a.nz, a.nzp));
  }
  a.out[idx] = v;
}

// Generic lengths, step 3: multiply the z spectra by H(kz).
__global__ void __launch_bounds__(kThreads) k_synt_filter(const __grid_constant__ SyntArgs a) {
  const long long plane = (long long)a.cnxp * a.nyp;
  const long long n = plane * a.nzp;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n) return;
  a.out[idx] = cmul(a.out[idx], __ldg(a.H + idx / plane));
}

// Generic lengths, step 5: traces outside x < nx, y < ny get imp back.
__global__ void __launch_bounds__(kThreads) k_synt_fixup(const __grid_constant__ SyntArgs a) {
  const long long plane = (long long)a.cnxp * a.nyp;
  const long long n = plane * a.nzp;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n) return;
  const long long col = idx % plane;
  const int y = (int)(col / a.cnxp), p = (int)(col % a.cnxp);
  const bool fx = 2 * p < a.nx, fy = 2 * p + 1 < a.nx;
  if (y < a.ny && fx && fy) return;
  const float2 raw = imp_at(a, idx);
  float2 v = a.out[idx];
  if (y >= a.ny || !fx) v.x = raw.x;
  if (y >= a.ny || !fy) v.y = raw.y;
  a.out[idx] = v;
}

template <int N>
int launch_synt(const SyntArgs &a, cudaStream_t s) {
  constexpr int TX = 8;
  const size_t smem = sizeof(float2) * (N + (size_t)cols_pitch(TX) * padded_rows(N, cols_padr(N, TX)));
  int rc = func_smem((const void *)k_synt<N, TX>, smem);
  if (rc) return rc;
  const dim3 grd((unsigned)((a.cnxp + TX - 1) / TX), (unsigned)a.nyp);
  k_synt<N, TX><<<grd, kThreads, smem, s>>>(a);
  CRAVA_LAUNCH_CHECK();
  return CRAVA_GPU_OK;
}

// H_l(kz) = D(kz) conj(W_l(kz)) / nzp in double, stored as float2 [nt][nzp];
// the upper half is the exact conjugate mirror of the lower, and the kz = 0
// and Nyquist entries are real (a real-to-complex inverse drops their
// imaginary parts).
std::vector<float2> synt_filters(const crava_gpu_ctx *c) {
  const int nzp = c->p.nzp, nt = c->p.ntheta;
  std::vector<float2> H((size_t)nt * nzp);
  for (int l = 0; l < nt; ++l) {
    const float *w = c->wavelet.data() + (size_t)l * nzp;
    for (int k = 0; 2 * k <= nzp; ++k) {
      double wr = 0.0, wi = 0.0;
      for (int n = 0; n < nzp; ++n) {
        const long long m = ((long long)k * n) % nzp;
        const double ang = -2.0 * M_PI * (double)m / nzp;
        wr += w[n] * cos(ang);
        wi += w[n] * sin(ang);
      }
      const double ang = 2.0 * M_PI * (double)k / nzp;
      const double dr = cos(ang) - 1.0, di = sin(ang);
      double hr = (dr * wr + di * wi) / nzp, hi = (di * wr - dr * wi) / nzp;
      if (k == 0 || 2 * k == nzp) hi = 0.0;
      H[(size_t)l * nzp + k] = make_float2((float)hr, (float)hi);
      if (k > 0 && 2 * k < nzp) H[(size_t)l * nzp + nzp - k] = make_float2((float)hr, -(float)hi);
    }
  }
  return H;
}

// Synthetic seismic with local wavelets, first step: every angle's
// impedance imp_l = A_l0 alpha + A_l1 beta + A_l2 rho on every cell (the
// reference's float sequence), and on the simbox traces (x < nx, y < ny)
// the tapered trace differenced forward in z (cyclic), the time-domain
// input of the per-trace wavelet filter (src/crava.cpp:1674-1694).  One
// thread per padded trace, x fastest; the three parameter grids are read
// once for all angles.
struct DiffArgs {
  const float *m[3];
  float *out[CRAVA_GPU_MAX_THETA];
  float A[CRAVA_GPU_MAX_THETA][3];
  int rnxp, nyp, nzp, nx, ny, nz;
};

template <int NT>
__global__ void __launch_bounds__(kThreads) k_synt_diff(const __grid_constant__ DiffArgs a) {
  const long long plane = (long long)a.rnxp * a.nyp;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= plane) return;
  const int i = (int)(t % a.rnxp), j = (int)(t / a.rnxp);
  auto imp = [&](int z, int l) {
    const long long o = t + (long long)z * plane;
    return imp1(a.m[0][o], a.m[1][o], a.m[2][o], a.A[l]);
  };
  if (!(i < a.nx && j < a.ny)) {
    for (int z = 0; z < a.nzp; ++z) {
      const long long o = t + (long long)z * plane;
      const float x = a.m[0][o], y = a.m[1][o], w = a.m[2][o];
#pragma unroll
      for (int l = 0; l < NT; ++l) a.out[l][o] = imp1(x, y, w, a.A[l]);
    }
    return;
  }
  // fac ((k - nz) imp[0] + (nzp - k - 1) imp[nz - 1]), fac = 1 / (nzp - nz - 1)
  const float fac = a.nz < a.nzp ? __fdiv_rn(1.0f, (float)(a.nzp - a.nz - 1)) : 0.0f;
  float v0[NT], vl[NT], prev[NT];
#pragma unroll
  for (int l = 0; l < NT; ++l) {
    v0[l] = imp(0, l);
    vl[l] = imp(a.nz - 1, l);
    prev[l] = v0[l];
  }
  for (int z = 0; z + 1 < a.nzp; ++z) {
    const int k = z + 1;
    float x = 0.f, y = 0.f, w = 0.f;
    if (k < a.nz) {
      const long long o = t + (long long)k * plane;
      x = a.m[0][o]; y = a.m[1][o]; w = a.m[2][o];
    }
    const long long oz = t + (long long)z * plane;
#pragma unroll
    for (int l = 0; l < NT; ++l) {
      const float next = k < a.nz ? imp1(x, y, w, a.A[l])
                                  : __fmul_rn(fac, __fadd_rn(__fmul_rn((float)(k - a.nz), v0[l]),
                                                             __fmul_rn((float)(a.nzp - k - 1), vl[l])));
      a.out[l][oz] = __fsub_rn(next, prev[l]);
      prev[l] = next;
    }
  }
  const long long ol = t + (long long)(a.nzp - 1) * plane;
#pragma unroll
  for (int l = 0; l < NT; ++l) a.out[l][ol] = __fsub_rn(v0[l], prev[l]);
}

}  // namespace

extern "C" int crava_gpu_synt_seismic(crava_gpu_ctx *c, const float *alpha, const float *beta,
                                      const float *rho, int nx, int ny, float *const *out) {
  if (!c || !alpha || !beta || !rho || !out) return CRAVA_GPU_ERR_ARG;
  const int nt = c->p.ntheta;
  auto mis = [](const void *p) { return !p || (reinterpret_cast<uintptr_t>(p) & 7u) != 0; };
  if (mis(alpha) || mis(beta) || mis(rho)) return CRAVA_GPU_ERR_ARG;
  for (int l = 0; l < nt; ++l) if (mis(out[l])) return CRAVA_GPU_ERR_ARG;
  if (nx == 0) nx = c->g.nxp;
  if (ny == 0) ny = c->g.nyp;
  const int nz = c->p.nz;
  if (nx < 1 || nx > c->g.nxp || ny < 1 || ny > c->g.nyp || nz < 1 || nz > c->g.nzp) return CRAVA_GPU_ERR_ARG;
  // the taper factor 1 / (nzp - nz - 1) is undefined with one padding layer
  if (nz == c->g.nzp - 1) return CRAVA_GPU_ERR_ARG;
  DeviceGuard guard(c->device);
  if (!c->synt_H) {
    std::vector<float2> H = synt_filters(c);
    if (cudaMalloc(&c->synt_H, H.size() * sizeof(float2)) != cudaSuccess) { c->synt_H = nullptr; return CRAVA_GPU_ERR_ALLOC; }
    CRAVA_CUDA_TRY(cudaMemcpy(c->synt_H, H.data(), H.size() * sizeof(float2), cudaMemcpyHostToDevice));
  }
  SyntArgs a{};
  a.m[0] = reinterpret_cast<const float2 *>(alpha);
  a.m[1] = reinterpret_cast<const float2 *>(beta);
  a.m[2] = reinterpret_cast<const float2 *>(rho);
  a.cnxp = c->g.cnxp; a.nyp = c->g.nyp; a.nzp = c->g.nzp;
  a.nx = nx; a.ny = ny; a.nz = nz;
  a.tw = c->plans.z.tw;
  const cudaStream_t s = c->stream;
  const long long n = c->g.csize;
  const dim3 eg((unsigned)((n + kThreads - 1) / kThreads));
  int rc;
  if (c->g.nzp == 128 || c->g.nzp == 256 || c->g.nzp == 512) {
    SyntAllArgs b{};
    for (int q = 0; q < 3; ++q) b.m[q] = a.m[q];
    for (int l = 0; l < nt; ++l) {
      b.out[l] = reinterpret_cast<float2 *>(out[l]);
      for (int q = 0; q < 3; ++q) b.A[l][q] = c->A[3 * l + q];
    }
    b.H = c->synt_H;
    b.tw = a.tw;
    b.nt = nt; b.cnxp = a.cnxp; b.nyp = a.nyp; b.nzp = a.nzp; b.nx = nx; b.ny = ny; b.nz = nz;
    switch (c->g.nzp) {
      case 128: return launch_synt_all<128>(b, s);
      case 256: return launch_synt_all<256>(b, s);
      default: return launch_synt_all<512>(b, s);
    }
  }
  for (int l = 0; l < nt; ++l) {
    a.out = reinterpret_cast<float2 *>(out[l]);
    a.H = c->synt_H + (size_t)l * c->g.nzp;
    for (int q = 0; q < 3; ++q) a.A[q] = c->A[3 * l + q];
    switch (c->g.nzp) {
      case 64: rc = launch_synt<64>(a, s); break;
      case 128: rc = launch_synt<128>(a, s); break;
      case 256: rc = launch_synt<256>(a, s); break;
      case 512: rc = launch_synt<512>(a, s); break;
      case 96: rc = launch_synt<96>(a, s); break;
      case 160: rc = launch_synt<160>(a, s); break;
      case 192: rc = launch_synt<192>(a, s); break;
      case 200: rc = launch_synt<200>(a, s); break;
      case 300: rc = launch_synt<300>(a, s); break;
      case 384: rc = launch_synt<384>(a, s); break;
      default: {
        k_synt_imp<<<eg, kThreads, 0, s>>>(a);
        CRAVA_LAUNCH_CHECK();
        if ((rc = fft_cols_z(c->plans, a.out, -1, s))) return rc;
        k_synt_filter<<<eg, kThreads, 0, s>>>(a);
        CRAVA_LAUNCH_CHECK();
        if ((rc = fft_cols_z(c->plans, a.out, 1, s))) return rc;
        k_synt_fixup<<<eg, kThreads, 0, s>>>(a);
        CRAVA_LAUNCH_CHECK();
        rc = CRAVA_GPU_OK;
      }
    }
    if (rc) return rc;
  }
  return CRAVA_GPU_OK;
}

extern "C" int crava_gpu_synt_seismic_local(crava_gpu_ctx *c, const float *alpha, const float *beta,
                                            const float *rho, int nx, int ny, const double *rel_thick,
                                            float dz, const float *shift, const float *gain, float *const *out) {
  if (!c || !alpha || !beta || !rho || !out || !rel_thick || !(dz > 0.0f)) return CRAVA_GPU_ERR_ARG;
  const int nt = c->p.ntheta;
  auto mis = [](const void *p) { return !p || (reinterpret_cast<uintptr_t>(p) & 7u) != 0; };
  if (mis(alpha) || mis(beta) || mis(rho)) return CRAVA_GPU_ERR_ARG;
  for (int l = 0; l < nt; ++l) if (mis(out[l])) return CRAVA_GPU_ERR_ARG;
  if (nx == 0) nx = c->g.nxp;
  if (ny == 0) ny = c->g.nyp;
  const int nz = c->p.nz;
  if (nx < 1 || nx > c->g.nxp || ny < 1 || ny > c->g.nyp || nz < 1 || nz > c->g.nzp) return CRAVA_GPU_ERR_ARG;
  if (nz == c->g.nzp - 1) return CRAVA_GPU_ERR_ARG;  // the taper divides by nzp - nz - 1
  DeviceGuard guard(c->device);
  DiffArgs a{};
  a.m[0] = alpha; a.m[1] = beta; a.m[2] = rho;
  for (int l = 0; l < nt; ++l) {
    a.out[l] = out[l];
    for (int q = 0; q < 3; ++q) a.A[l][q] = c->A[3 * l + q];
  }
  a.rnxp = c->g.rnxp; a.nyp = c->g.nyp; a.nzp = c->g.nzp; a.nx = nx; a.ny = ny; a.nz = nz;
  const long long ntr = (long long)a.rnxp * a.nyp;
  const dim3 grd((unsigned)((ntr + kThreads - 1) / kThreads));
  const cudaStream_t s = c->stream;
  switch (nt) {
#define CRAVA_DIFF_CASE(N) case N: k_synt_diff<N><<<grd, kThreads, 0, s>>>(a); break;
    CRAVA_DIFF_CASE(1) CRAVA_DIFF_CASE(2) CRAVA_DIFF_CASE(3) CRAVA_DIFF_CASE(4)
    CRAVA_DIFF_CASE(5) CRAVA_DIFF_CASE(6) CRAVA_DIFF_CASE(7) CRAVA_DIFF_CASE(8)
#undef CRAVA_DIFF_CASE
    default: return CRAVA_GPU_ERR_ARG;
  }
  CRAVA_LAUNCH_CHECK();
  // resultVec.fft1DInPlace(), times conj(localWavelet->getCAmp(k, sf)),
  // invFFT1DInPlace() (1 / nzp): the per-trace filter of the multiply-back
  // with no pre-scale and 1 / nzp after
  return multiply_local_wavelet(c, out, rel_thick, nx, ny, dz, shift, gain, 1.0f, (float)c->g.nzp, false);
}
