// fft.cu -- 3-D real<->complex transforms on the reference's padded layout.
//
// Replaces FFTGrid::fftInPlace / invFFTInPlace (src/fftgrid.cpp:1803-1862),
// which call FFTW 2.1.2's rfftw3d (real-to-half-complex along x, complex
// along y and z, unnormalised, forward sign -) and scale by 1/sqrt(N)
// (DATA, PARAMETER) or 1 forward / 1/N inverse (COVARIANCE).
//
// Three passes, each one read and one write of the grid:
//   rows  (x): each CTA transforms ROWS rows of nxp reals; an even nxp is
//              done as one nxp/2-point complex FFT of the packed row and a
//              split step (the row's float pairs are read as float2).
//   cols  (y): each CTA transforms TX adjacent x-columns of one z-plane.
//   cols  (z): each CTA transforms TX adjacent x-columns of one y-row.
// Lines live in shared memory and go through the Stockham engine of
// fft_core.cuh; at the power-of-two lengths 64..512 the register-resident
// passes of fft_rr.cuh are the default (same arithmetic, fewer shared-memory
// round trips).  The scalings are fused into the first (forward) or last
// (inverse) pass.
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include <vector>

#include "fft.cuh"
#include "fft_core.cuh"
#include "fft_rr.cuh"

namespace crava {

namespace {

constexpr int kThreads = 256;
constexpr int kRows = 16;    // rows per CTA in the x pass
constexpr int kColTile = 8;  // x-columns per CTA in the y / z passes

struct RowArgs {
  float *grid;
  const float *src;  // forward: input grid (may equal grid)
  long long nrows;  // nyp * nzp
  int rnxp;         // floats per row
  int nxp;
  RadixList rl;     // line length: nxp/2 (even) or nxp (odd)
  const float2 *tw;
  const float2 *post;  // e^{-2 pi i k/nxp}, k <= nxp/2 (even nxp)
  const float *addend; // inverse only: real grid added to the output (or null)
  float scale;
};

struct ColArgs {
  float2 *data;
  int ninner;              // cnxp
  long long elem_stride;   // between consecutive line elements (float2)
  long long outer_stride;  // between CTAs along blockIdx.y (float2)
  RadixList rl;
  const float2 *tw;
  float scale;
};

// ------------------------------------------------------------------ x pass
template <int DIR, bool EVEN>
__global__ void __launch_bounds__(kThreads) k_rows(const __grid_constant__ RowArgs a) {
  extern __shared__ float2 sm[];
  const int n = a.rl.n;            // complex line length
  const int ld = n + 1;            // shared row pitch
  float2 *twl = sm;                // n
  float2 *post = twl + n;          // n + 1 (even only)
  float2 *bufA = post + (EVEN ? n + 1 : 0);
  float2 *bufB = bufA + kRows * ld;
  const long long row0 = (long long)blockIdx.x * kRows;
  const int nrows = (int)min((long long)kRows, a.nrows - row0);
  const int tid = threadIdx.x;
  for (int i = tid; i < n; i += blockDim.x) twl[i] = a.tw[i];
  if (EVEN)
    for (int i = tid; i <= n; i += blockDim.x) post[i] = a.post[i];
  __syncthreads();

  if (DIR < 0) {
    // forward: load (asynchronous copies for an even row; the scale is
    // applied after the transform)
    for (int idx = tid; idx < kRows * n; idx += blockDim.x) {
      int r = idx / n, m = idx % n;
      if (r < nrows) {
        const float *row = a.src + (row0 + r) * a.rnxp;
        if (EVEN) cp_async8(bufA + r * ld + m, reinterpret_cast<const float2 *>(row) + m);
        else bufA[r * ld + m] = make_float2(__ldg(row + m), 0.f);
      } else {
        bufA[r * ld + m] = make_float2(0.f, 0.f);
      }
    }
    cp_async_wait_all();
  } else {
    // inverse: load the half spectrum and build the line to transform
    for (int idx = tid; idx < kRows * n; idx += blockDim.x) {
      int r = idx / n, k = idx % n;
      float2 v = make_float2(0.f, 0.f);
      if (r < nrows) {
        const float2 *X = reinterpret_cast<const float2 *>(a.grid + (row0 + r) * a.rnxp);
        if (EVEN) {
          // Z'[k] = (X_k + conj X_{h-k}) + i W^{-k} (X_k - conj X_{h-k}),
          // imaginary parts of DC and Nyquist ignored.
          float2 xk = X[k], xm = X[n - k];
          if (k == 0) { xk.y = 0.f; xm.y = 0.f; }
          xm.y = -xm.y;
          float2 e = cadd(xk, xm);
          float2 w = post[k];
          w.y = -w.y;  // W^{-k}
          float2 o = cmul(csub(xk, xm), w);
          v = make_float2(e.x - o.y, e.y + o.x);
        } else {
          const int c = n / 2 + 1;
          if (k == 0) v = make_float2(X[0].x, 0.f);
          else if (k < c) v = X[k];
          else { v = X[n - k]; v.y = -v.y; }
        }
      }
      bufA[r * ld + k] = v;
    }
  }
  __syncthreads();
  int which = stockham<DIR, false>(bufA, ld, 1, bufB, ld, 1, a.rl, twl, kRows);
  const float2 *res = which ? bufB : bufA;

  if (DIR < 0) {
    if (EVEN) {
      // X_k = E_k + W^k O_k, E = (Z_k + conj Z_{h-k})/2, O = -i (Z_k - conj Z_{h-k})/2
      for (int idx = tid; idx < kRows * (n + 1); idx += blockDim.x) {
        int r = idx / (n + 1), k = idx % (n + 1);
        if (r >= nrows) continue;
        float2 zk = res[r * ld + (k == n ? 0 : k)];
        float2 zm = res[r * ld + (k == 0 ? 0 : n - k)];
        zm.y = -zm.y;
        float2 e = cscale(cadd(zk, zm), 0.5f);
        float2 d = csub(zk, zm);
        float2 o = make_float2(0.5f * d.y, -0.5f * d.x);
        float2 X = cadd(e, cmul(post[k], o));
        reinterpret_cast<float2 *>(a.grid + (row0 + r) * a.rnxp)[k] = cscale(X, a.scale);
      }
    } else {
      const int c = n / 2 + 1;
      for (int idx = tid; idx < kRows * c; idx += blockDim.x) {
        int r = idx / c, k = idx % c;
        if (r >= nrows) continue;
        reinterpret_cast<float2 *>(a.grid + (row0 + r) * a.rnxp)[k] = cscale(res[r * ld + k], a.scale);
      }
    }
  } else {
    if (EVEN) {
      for (int idx = tid; idx < kRows * (n + 1); idx += blockDim.x) {
        int r = idx / (n + 1), m = idx % (n + 1);
        if (r >= nrows) continue;
        float2 v = make_float2(0.f, 0.f);
        if (m < n) {
          v = cscale(res[r * ld + m], a.scale);
          if (a.addend) v = cadd(v, reinterpret_cast<const float2 *>(a.addend + (row0 + r) * a.rnxp)[m]);
        }
        reinterpret_cast<float2 *>(a.grid + (row0 + r) * a.rnxp)[m] = v;
      }
    } else {
      for (int idx = tid; idx < kRows * (n + 1); idx += blockDim.x) {
        int r = idx / (n + 1), m = idx % (n + 1);
        if (r >= nrows) continue;
        float v = 0.f;
        if (m < n) {
          v = res[r * ld + m].x * a.scale;
          if (a.addend) v += a.addend[(row0 + r) * a.rnxp + m];
        }
        a.grid[(row0 + r) * a.rnxp + m] = v;
      }
    }
  }
}

// ------------------------------------------------------------------ y / z pass
template <int DIR>
__global__ void __launch_bounds__(kThreads) k_cols(const __grid_constant__ ColArgs a) {
  extern __shared__ float2 sm[];
  const int n = a.rl.n;
  float2 *twl = sm;
  float2 *bufA = twl + n;
  float2 *bufB = bufA + kColTile * n;
  const int x0 = blockIdx.x * kColTile;
  const int nx = min(kColTile, a.ninner - x0);
  float2 *base = a.data + (long long)blockIdx.y * a.outer_stride + x0;
  const int tid = threadIdx.x;
  for (int i = tid; i < n; i += blockDim.x) twl[i] = a.tw[i];
  for (int idx = tid; idx < kColTile * n; idx += blockDim.x) {
    int t = idx % kColTile, m = idx / kColTile;
    if (t < nx) cp_async8(bufA + m * kColTile + t, base + m * a.elem_stride + t);
    else bufA[m * kColTile + t] = make_float2(0.f, 0.f);
  }
  cp_async_wait_all();
  __syncthreads();
  int which = stockham<DIR, true>(bufA, 1, kColTile, bufB, 1, kColTile, a.rl, twl, kColTile);
  const float2 *res = which ? bufB : bufA;
  for (int idx = tid; idx < kColTile * n; idx += blockDim.x) {
    int t = idx % kColTile, m = idx / kColTile;
    if (t < nx) base[m * a.elem_stride + t] = cscale(res[m * kColTile + t], a.scale);
  }
}

// The same column pass with the line length N a compile-time constant.
template <int N, int DIR>
__global__ void __launch_bounds__(kThreads) k_cols_ct(const __grid_constant__ ColArgs a) {
  extern __shared__ float2 sm[];
  float2 *twl = sm;
  float2 *bufA = twl + N;
  float2 *bufB = bufA + kColTile * N;
  const int x0 = blockIdx.x * kColTile;
  const int nx = min(kColTile, a.ninner - x0);
  float2 *base = a.data + (long long)blockIdx.y * a.outer_stride + x0;
  const int tid = threadIdx.x;
  for (int i = tid; i < N; i += blockDim.x) twl[i] = a.tw[i];
  for (int idx = tid; idx < kColTile * N; idx += blockDim.x) {
    int t = idx % kColTile, m = idx / kColTile;
    if (t < nx) cp_async8(bufA + m * kColTile + t, base + m * a.elem_stride + t);
    else bufA[m * kColTile + t] = make_float2(0.f, 0.f);
  }
  cp_async_wait_all();
  __syncthreads();
  const int which = stockham_ct<N, DIR, true, kColTile, 1, kColTile, 1, kColTile>(bufA, bufB, twl);
  const float2 *res = which ? bufB : bufA;
  for (int idx = tid; idx < kColTile * N; idx += blockDim.x) {
    int t = idx % kColTile, m = idx / kColTile;
    if (t < nx) base[m * a.elem_stride + t] = cscale(res[m * kColTile + t], a.scale);
  }
}

// Row (x) pass for an even nxp, N = nxp / 2 a compile-time constant, in
// place: RR rows per CTA held element-major ([m][r], odd pitch RR + 1).
constexpr int kRR = 32;
template <int N, int DIR>
__global__ void __launch_bounds__(kThreads) k_rows_ip(const __grid_constant__ RowArgs a) {
  constexpr int P = kRR + 1;
  extern __shared__ float2 sm[];
  float2 *twl = sm;            // N
  float2 *post = twl + N;      // N + 1
  float2 *buf = post + N + 1;  // N * P
  const long long row0 = (long long)blockIdx.x * kRR;
  const int nrows = (int)min((long long)kRR, a.nrows - row0);
  const int tid = threadIdx.x;
  for (int i = tid; i < N; i += kThreads) twl[i] = a.tw[i];
  for (int i = tid; i <= N; i += kThreads) post[i] = a.post[i];
  // One warp per row, lanes along the row: each thread issues all its
  // loads (RPW rows x C columns) before the first use.
  const int warp = tid >> 5, lane = tid & 31;
  constexpr int NW = kThreads / 32;
  constexpr int RPW = (kRR + NW - 1) / NW;
  constexpr int C = (N + 31) / 32;
  if (DIR < 0) {
    float2 v[RPW][C];
#pragma unroll
    for (int i = 0; i < RPW; ++i) {
      const int r = warp + i * NW;
      const float2 *row = reinterpret_cast<const float2 *>(a.src + (row0 + r) * a.rnxp);
#pragma unroll
      for (int c = 0; c < C; ++c) {
        const int m = lane + 32 * c;
        v[i][c] = (r < nrows && m < N) ? row[m] : make_float2(0.f, 0.f);
      }
    }
#pragma unroll
    for (int i = 0; i < RPW; ++i) {
      const int r = warp + i * NW;
#pragma unroll
      for (int c = 0; c < C; ++c) {
        const int m = lane + 32 * c;
        if (r < kRR && m < N) buf[m * P + r] = v[i][c];
      }
    }
  } else {
    __syncthreads();
    // Z'[k] = (X_k + conj X_{h-k}) + i W^{-k} (X_k - conj X_{h-k}); the
    // imaginary parts of DC and Nyquist are ignored, as a C2R does.
    float2 xk[RPW][C], xm[RPW][C];
#pragma unroll
    for (int i = 0; i < RPW; ++i) {
      const int r = warp + i * NW;
      const float2 *X = reinterpret_cast<const float2 *>(a.grid + (row0 + r) * a.rnxp);
#pragma unroll
      for (int c = 0; c < C; ++c) {
        const int k = lane + 32 * c;
        if (r < nrows && k < N) {
          xk[i][c] = X[k];
          xm[i][c] = X[N - k];
        } else {
          xk[i][c] = xm[i][c] = make_float2(0.f, 0.f);
        }
      }
    }
#pragma unroll
    for (int i = 0; i < RPW; ++i) {
      const int r = warp + i * NW;
#pragma unroll
      for (int c = 0; c < C; ++c) {
        const int k = lane + 32 * c;
        if (r >= kRR || k >= N) continue;
        float2 x0 = xk[i][c], x1 = xm[i][c];
        if (k == 0) { x0.y = 0.f; x1.y = 0.f; }
        x1.y = -x1.y;
        const float2 e = cadd(x0, x1);
        float2 w = post[k];
        w.y = -w.y;
        const float2 o = cmul(csub(x0, x1), w);
        buf[k * P + r] = make_float2(e.x - o.y, e.y + o.x);
      }
    }
  }
  __syncthreads();
  stockham_ip<N, DIR, kRR, 1, P, kThreads>(buf, twl);
  // Output loops, one warp per row as well: no division by the row length
  // (N + 1 outputs) and one row address per warp and row.
  if (DIR < 0) {
    // X_k = E_k + W^k O_k, E = (Z_k + conj Z_{h-k})/2, O = -i (Z_k - conj Z_{h-k})/2
    for (int r = warp; r < nrows; r += kThreads / 32) {
      float2 *orow = reinterpret_cast<float2 *>(a.grid + (row0 + r) * a.rnxp);
      for (int k = lane; k <= N; k += 32) {
        const float2 zk = buf[(k == N ? 0 : k) * P + r];
        float2 zm = buf[(k == 0 ? 0 : N - k) * P + r];
        zm.y = -zm.y;
        const float2 e = cscale(cadd(zk, zm), 0.5f);
        const float2 d = csub(zk, zm);
        const float2 o = make_float2(0.5f * d.y, -0.5f * d.x);
        orow[k] = cscale(cadd(e, cmul(post[k], o)), a.scale);
      }
    }
  } else {
    for (int r = warp; r < nrows; r += kThreads / 32) {
      float2 *orow = reinterpret_cast<float2 *>(a.grid + (row0 + r) * a.rnxp);
      const float2 *arow = a.addend ? reinterpret_cast<const float2 *>(a.addend + (row0 + r) * a.rnxp) : nullptr;
      for (int m = lane; m <= N; m += 32) {
        float2 v = make_float2(0.f, 0.f);
        if (m < N) {
          v = cscale(buf[m * P + r], a.scale);
          if (arow) v = cadd(v, arow[m]);
        }
        orow[m] = v;
      }
    }
  }
}

// Column pass, in-place register-staged transform, TX columns per CTA.
template <int N, int DIR, int TX>
__global__ void __launch_bounds__(kThreads) k_cols_ip(const __grid_constant__ ColArgs a) {
  extern __shared__ float2 sm[];
  float2 *twl = sm;
  float2 *buf = twl + N;
  const int x0 = blockIdx.x * TX;
  const int nx = min(TX, a.ninner - x0);
  float2 *base = a.data + (long long)blockIdx.y * a.outer_stride + x0;
  const int tid = threadIdx.x;
  constexpr int ES = cols_pitch(TX);
  constexpr int PADR = cols_padr(N, TX);
  for (int i = tid; i < N; i += kThreads) twl[i] = a.tw[i];
  for (int idx = tid; idx < TX * N; idx += kThreads) {
    const int t = idx % TX, m = idx / TX;
    float2 *dst = buf + pad_row<PADR>(m) * ES + t;
    if (t < nx) cp_async8(dst, base + m * a.elem_stride + t);
    else *dst = make_float2(0.f, 0.f);
  }
  cp_async_wait_all();
  __syncthreads();
  stockham_ip<N, DIR, TX, 1, ES, kThreads, PADR>(buf, twl);
  for (int idx = tid; idx < TX * N; idx += kThreads) {
    const int t = idx % TX, m = idx / TX;
    if (t < nx) base[m * a.elem_stride + t] = cscale(buf[pad_row<PADR>(m) * ES + t], a.scale);
  }
}

// ------------------------------------------------------------------ register-resident passes
// (fft_rr.cuh).  Column pass: kRrTX lines per CTA; line f starts at
// base(f) = (f mod A) + (f div A) B and its elements are es apart:
//   z pass: A = the line count, B = 0  -> base = f, es = cnxp nyp
//           (the lines of a z plane taken flat: no ragged tiles);
//   y pass: A = cnxp, B = cnxp nyp     -> lines (kx, z), es = cnxp.
// CPT lines per thread (2: a float4 shared-memory row access carries both);
// shared rows hold kRrTX float2 = 128 B, so a phase of 8 (float4) or 16
// (float2) lanes covers exactly one row: no bank conflicts whatever the
// stage's index pattern.  VEC: the two lines of a thread are adjacent and
// 16-byte aligned in global memory (z pass, even es), loaded as one float4.
constexpr int kRrTX = 16;

struct ColRRArgs {
  float2 *data;
  long long nlines;
  FastDiv fa;
  uint32_t A;
  long long B;
  long long es;
  const float2 *tw;
  ZPrior zp;  // forward z pass of a covariance grid: the band-gated rule (inv null: none)
};

template <int N>
struct RrCols {
  static constexpr int E = rr::max_radix(N);
  static constexpr int T = N / E;
  static constexpr int CPT = E >= 16 ? 1 : 2;
  static constexpr int NP = kRrTX / CPT;
  static constexpr int NTH = NP * T;
};

template <int N, int DIR, int CPT, bool VEC, int S>
struct RrColStages {
  // v holds the inputs of stage S (registers (b, q) of radix R_S)
  static __device__ __forceinline__ void run(float2 (&v)[CPT][RrCols<N>::E], float2 *buf,
                                             const float2 *tw, int t, int p, float2 *const *gp,
                                             long long es, const bool *ok, const ZPrior &zp,
                                             const float2 *base, unsigned gmask) {
    constexpr int E = RrCols<N>::E, T = RrCols<N>::T, R = CtRadix::at(N, S);
#pragma unroll
    for (int c = 0; c < CPT; ++c) rr::stage_compute<N, S, DIR, E, T>(v[c], tw, t);
    if constexpr (S + 1 == CtRadix::count(N)) {
      // last stage: outputs at the loaded positions, straight to HBM
      if (DIR < 0 && gmask) {
        // band-gated kz planes of a covariance grid (gmask: this thread's
        // output registers on them): the prior rule
#pragma unroll
        for (int b = 0; b < E / R; ++b)
#pragma unroll
          for (int q = 0; q < R; ++q) {
            if ((gmask >> (b * R + q)) & 1u) {
              const int e = rr::stage_in<N, S, E, T>(t, b, q);
#pragma unroll
              for (int c = 0; c < CPT; ++c)
                if (ok[c]) v[c][b * R + q] = zprior_apply(zp, v[c][b * R + q], (long long)(gp[c] - base) + (long long)e * es);
            }
          }
      }
#pragma unroll
      for (int b = 0; b < E / R; ++b)
#pragma unroll
        for (int q = 0; q < R; ++q) {
          const long long e = rr::stage_in<N, S, E, T>(t, b, q);
          if (VEC) {
            if (ok[0])
              *reinterpret_cast<float4 *>(gp[0] + e * es) =
                  make_float4(v[0][b * R + q].x, v[0][b * R + q].y, v[CPT - 1][b * R + q].x, v[CPT - 1][b * R + q].y);
          } else {
#pragma unroll
            for (int c = 0; c < CPT; ++c)
              if (ok[c]) gp[c][e * es] = v[c][b * R + q];
          }
        }
    } else {
      if (S > 0) __syncthreads();  // every thread has read this stage's inputs
#pragma unroll
      for (int b = 0; b < E / R; ++b)
#pragma unroll
        for (int q = 0; q < R; ++q) {
          const int o = rr::stage_out<N, S, T>(t, b, q);
          if (CPT == 2)
            *reinterpret_cast<float4 *>(buf + o * kRrTX + 2 * p) =
                make_float4(v[0][b * R + q].x, v[0][b * R + q].y, v[CPT - 1][b * R + q].x, v[CPT - 1][b * R + q].y);
          else
            buf[o * kRrTX + p] = v[0][b * R + q];
        }
      __syncthreads();
      constexpr int R2 = CtRadix::at(N, S + 1);
#pragma unroll
      for (int b = 0; b < E / R2; ++b)
#pragma unroll
        for (int q = 0; q < R2; ++q) {
          const int e = rr::stage_in<N, S + 1, E, T>(t, b, q);
          if (CPT == 2) {
            const float4 x = *reinterpret_cast<const float4 *>(buf + e * kRrTX + 2 * p);
            v[0][b * R2 + q] = make_float2(x.x, x.y);
            v[CPT - 1][b * R2 + q] = make_float2(x.z, x.w);
          } else {
            v[0][b * R2 + q] = buf[e * kRrTX + p];
          }
        }
      RrColStages<N, DIR, CPT, VEC, S + 1>::run(v, buf, tw, t, p, gp, es, ok, zp, base, gmask);
    }
  }
};

template <int N, int DIR, bool VEC>
__global__ void __launch_bounds__(RrCols<N>::NTH) k_cols_rr(const __grid_constant__ ColRRArgs a) {
  using C = RrCols<N>;
  constexpr int E = C::E, T = C::T, CPT = C::CPT, NP = C::NP;
  constexpr int R0 = CtRadix::at(N, 0);
  extern __shared__ float4 sm4[];
  float2 *tw = reinterpret_cast<float2 *>(sm4);
  float2 *buf = tw + N;  // [N][kRrTX]
  const int tid = threadIdx.x;
  const int p = tid % NP, t = tid / NP;
  for (int i = tid; i < N; i += C::NTH) tw[i] = a.tw[i];
  float2 *gp[CPT];
  bool ok[CPT];
#pragma unroll
  for (int c = 0; c < CPT; ++c) {
    const long long f = (long long)blockIdx.x * kRrTX + p * CPT + c;
    ok[c] = f < a.nlines;
    const uint32_t q = ok[c] ? fdiv((uint32_t)f, a.fa) : 0u;
    const long long base = ok[c] ? (f - (long long)q * a.A) + (long long)q * a.B : 0;
    gp[c] = a.data + base;
  }
  float2 v[CPT][E];
#pragma unroll
  for (int b = 0; b < E / R0; ++b)
#pragma unroll
    for (int q = 0; q < R0; ++q) {
      const long long e = rr::stage_in<N, 0, E, T>(t, b, q);
      if (VEC) {
        const float4 x = ok[0] ? __ldg(reinterpret_cast<const float4 *>(gp[0] + e * a.es))
                               : make_float4(0.f, 0.f, 0.f, 0.f);
        v[0][b * R0 + q] = make_float2(x.x, x.y);
        v[CPT - 1][b * R0 + q] = make_float2(x.z, x.w);
      } else {
#pragma unroll
        for (int c = 0; c < CPT; ++c) v[c][b * R0 + q] = ok[c] ? gp[c][e * a.es] : make_float2(0.f, 0.f);
      }
    }
  __syncthreads();  // twiddles
  const unsigned gmask = DIR < 0 ? zprior_mask<N, E, T>(a.zp, t) : 0u;
  RrColStages<N, DIR, CPT, VEC, 0>::run(v, buf, tw, t, p, gp, a.es, ok, a.zp, a.data, gmask);
}

// Row (x) pass for an even nxp, N = nxp / 2, register-resident: ROWS
// rows per CTA (32, fewer when the CTA would exceed 512 threads), T threads
// per row (lanes along the row).  Forward: the
// packed row's N complex values go global -> registers, through the radix
// stages, to the split X_k = E_k + W^k O_k (which pairs k with N - k), and
// the N + 1 outputs to HBM.  Inverse: the pre-split Z'_k is built from X_k
// and X_{N-k}, and the last stage writes the real row straight to HBM.
// Where a row's T threads lie in one warp (T <= 32) the pairing is a warp
// shuffle; otherwise (N = 512) the split goes through shared memory and the
// pre-split reads X_{N-k} from HBM a second time.  Shared rows are padded
// (one spare element after every R_0 and a pitch of 8 mod 16 float2) so
// the first stage's stride-R_0 writes and two rows per phase are free of
// bank conflicts.
template <int N>
struct RrRows {
  static constexpr int E = rr::max_radix(N);
  static constexpr int T = N / E;
  static constexpr int ROWS = 512 / T < 32 ? 512 / T : 32;
  static constexpr int NTH = ROWS * T;
  static constexpr int R0 = CtRadix::at(N, 0);
  static constexpr int P0 = N + N / R0 + 1;  // room for index N in the split
  static constexpr int P = P0 + ((8 - P0 % 16) + 16) % 16;  // pitch = 8 mod 16
  static __host__ __device__ constexpr int phys(int e) { return e + e / R0; }
  // register holding position t + T m in stage s's layout (radix R):
  // b = m mod (E / R), q = m div (E / R), register b R + q
  static __host__ __device__ constexpr int reg(int m, int R) { return (m % (E / R)) * R + m / (E / R); }
  // A row's T threads are consecutive; with T <= 32 (a power of two) they
  // lie in one warp, and a warp barrier orders the row's shared-memory
  // exchanges (and its in-place global reads before writes); a row of
  // 64 threads spans two warps and takes the block barrier.
  static __device__ __forceinline__ void row_sync() {
    if constexpr (T <= 32) __syncwarp();
    else __syncthreads();
  }
};

template <int N, int DIR, int S>
struct RrRowStages {
  static __device__ __forceinline__ void run(float2 (&v)[RrRows<N>::E], float2 *row, const float2 *tw, int t) {
    constexpr int E = RrRows<N>::E, T = RrRows<N>::T, R = CtRadix::at(N, S);
    // the inverse reads its twiddles from the per-stage tables (measured
    // faster there; the forward is faster with the length-N table)
    if constexpr (DIR > 0) rr::stage_compute_st<N, S, DIR, E, T>(v, tw, t);
    else rr::stage_compute<N, S, DIR, E, T>(v, tw, t);
    if constexpr (S + 1 < CtRadix::count(N)) {
      if (S > 0) RrRows<N>::row_sync();
#pragma unroll
      for (int b = 0; b < E / R; ++b)
#pragma unroll
        for (int q = 0; q < R; ++q) row[RrRows<N>::phys(rr::stage_out<N, S, T>(t, b, q))] = v[b * R + q];
      RrRows<N>::row_sync();
      constexpr int R2 = CtRadix::at(N, S + 1);
#pragma unroll
      for (int b = 0; b < E / R2; ++b)
#pragma unroll
        for (int q = 0; q < R2; ++q) v[b * R2 + q] = row[RrRows<N>::phys(rr::stage_in<N, S + 1, E, T>(t, b, q))];
      RrRowStages<N, DIR, S + 1>::run(v, row, tw, t);
    }
  }
};

template <int N, int DIR>
__global__ void __launch_bounds__(RrRows<N>::NTH) k_rows_rr(const __grid_constant__ RowArgs a) {
  using C = RrRows<N>;
  constexpr int E = C::E, T = C::T, R0 = C::R0, S = CtRadix::count(N);
  constexpr int RL = CtRadix::at(N, S - 1);
  extern __shared__ float4 sm4[];
  float2 *tw = reinterpret_cast<float2 *>(sm4);  // twiddles (per-stage tables in the inverse)
  float2 *post = tw + rr::tw_slots<N>();          // N + 1
  float2 *buf = post + N + 1;                     // ROWS rows of pitch P
  const int tid = threadIdx.x;
  const int t = tid % T, r = tid / T;
  if constexpr (DIR > 0) {
    rr::tw_stages_fill<N>(tw, a.tw, tid, C::NTH);
  } else {
    for (int i = tid; i < N; i += C::NTH) tw[i] = a.tw[i];
  }
  for (int i = tid; i <= N; i += C::NTH) post[i] = a.post[i];
  const long long row_idx = (long long)blockIdx.x * C::ROWS + r;
  const bool ok = row_idx < a.nrows;
  float2 *row = buf + r * C::P;
  float2 v[E];
  if (DIR < 0) {
    const float2 *src = reinterpret_cast<const float2 *>(a.src + (ok ? row_idx : 0) * a.rnxp);
#pragma unroll
    for (int b = 0; b < E / R0; ++b)
#pragma unroll
      for (int q = 0; q < R0; ++q)
        v[b * R0 + q] = ok ? src[rr::stage_in<N, 0, E, T>(t, b, q)] : make_float2(0.f, 0.f);
    __syncthreads();  // twiddles
    RrRowStages<N, DIR, 0>::run(v, row, tw, t);
    if constexpr (T <= 32) {
      // the split pairs position k = t + T m with N - k, which thread
      // T - t of the same row holds at m' = E - 1 - m (thread 0: its own
      // position E - m): one warp shuffle per output instead of a
      // shared-memory round trip
      const int lane = threadIdx.x & 31;
      const int src = lane - t + (T - t) % T;
      float2 *orow = reinterpret_cast<float2 *>(a.grid + (ok ? row_idx : 0) * a.rnxp);
#pragma unroll
      for (int m = 0; m < E; ++m) {
        const float2 send = v[C::reg(E - 1 - m, RL)];
        float2 zm = make_float2(__shfl_sync(0xffffffffu, send.x, src), __shfl_sync(0xffffffffu, send.y, src));
        if (t == 0) zm = v[C::reg(m == 0 ? 0 : E - m, RL)];
        const float2 zk = v[C::reg(m, RL)];
        zm.y = -zm.y;
        const float2 e = cscale(cadd(zk, zm), 0.5f);
        const float2 d = csub(zk, zm);
        const float2 o = make_float2(0.5f * d.y, -0.5f * d.x);
        const int k = t + T * m;
        if (ok) orow[k] = cscale(cadd(e, cmul(post[k], o)), a.scale);
      }
      if (ok && t == 0) {
        // X_N from Z_0 alone
        const float2 zk = v[C::reg(0, RL)];
        float2 zm = zk;
        zm.y = -zm.y;
        const float2 e = cscale(cadd(zk, zm), 0.5f);
        const float2 d = csub(zk, zm);
        const float2 o = make_float2(0.5f * d.y, -0.5f * d.x);
        orow[N] = cscale(cadd(e, cmul(post[N], o)), a.scale);
      }
    } else {
      // last stage outputs to shared memory for the split
      if (S > 1) __syncthreads();
#pragma unroll
      for (int b = 0; b < E / RL; ++b)
#pragma unroll
        for (int q = 0; q < RL; ++q) row[C::phys(rr::stage_in<N, S - 1, E, T>(t, b, q))] = v[b * RL + q];
      __syncthreads();
      if (ok) {
        // X_k = E_k + W^k O_k, E = (Z_k + conj Z_{N-k})/2, O = -i (Z_k - conj Z_{N-k})/2
        float2 *orow = reinterpret_cast<float2 *>(a.grid + row_idx * a.rnxp);
        for (int k = t; k <= N; k += T) {
          const float2 zk = row[C::phys(k == N ? 0 : k)];
          float2 zm = row[C::phys(k == 0 ? 0 : N - k)];
          zm.y = -zm.y;
          const float2 e = cscale(cadd(zk, zm), 0.5f);
          const float2 d = csub(zk, zm);
          const float2 o = make_float2(0.5f * d.y, -0.5f * d.x);
          orow[k] = cscale(cadd(e, cmul(post[k], o)), a.scale);
        }
      }
    }
  } else {
    __syncthreads();  // twiddles and post
    const float2 *X = reinterpret_cast<const float2 *>(a.grid + (ok ? row_idx : 0) * a.rnxp);
    // Z'[k] = (X_k + conj X_{N-k}) + i W^{-k} (X_k - conj X_{N-k}); the
    // imaginary parts of DC and Nyquist are ignored, as a C2R does
    auto pre = [&](int k, float2 x0, float2 x1) {
      if (k == 0) { x0.y = 0.f; x1.y = 0.f; }
      x1.y = -x1.y;
      const float2 e = cadd(x0, x1);
      float2 w = post[k];
      w.y = -w.y;
      const float2 o = cmul(csub(x0, x1), w);
      return make_float2(e.x - o.y, e.y + o.x);
    };
    if constexpr (T <= 32) {
      // each thread loads its own positions k = t + T m; X_{N-k} comes
      // from thread T - t of the row by a warp shuffle (thread 0: its own
      // position E - m, and X_N, loaded once)
      float2 xk[E];
#pragma unroll
      for (int m = 0; m < E; ++m) xk[m] = ok ? X[t + T * m] : make_float2(0.f, 0.f);
      const float2 xN = (ok && t == 0) ? X[N] : make_float2(0.f, 0.f);
      const int lane = threadIdx.x & 31;
      const int src = lane - t + (T - t) % T;
#pragma unroll
      for (int m = 0; m < E; ++m) {
        const float2 send = xk[E - 1 - m];
        float2 x1 = make_float2(__shfl_sync(0xffffffffu, send.x, src), __shfl_sync(0xffffffffu, send.y, src));
        if (t == 0) x1 = m == 0 ? xN : xk[E - m];
        v[C::reg(m, R0)] = pre(t + T * m, xk[m], x1);
      }
    } else {
#pragma unroll
      for (int b = 0; b < E / R0; ++b)
#pragma unroll
        for (int q = 0; q < R0; ++q) {
          const int k = rr::stage_in<N, 0, E, T>(t, b, q);
          const float2 x0 = ok ? X[k] : make_float2(0.f, 0.f), x1 = ok ? X[N - k] : make_float2(0.f, 0.f);
          v[b * R0 + q] = pre(k, x0, x1);
        }
    }
    // every thread has read its whole row before any row is overwritten
    // (in place: the output row is the input row)
    if constexpr (T <= 32) __syncwarp();
    else __syncthreads();
    RrRowStages<N, DIR, 0>::run(v, row, tw, t);
    if (ok) {
      float2 *orow = reinterpret_cast<float2 *>(a.grid + row_idx * a.rnxp);
      const float2 *arow = a.addend ? reinterpret_cast<const float2 *>(a.addend + row_idx * a.rnxp) : nullptr;
#pragma unroll
      for (int b = 0; b < E / RL; ++b)
#pragma unroll
        for (int q = 0; q < RL; ++q) {
          const int m = rr::stage_in<N, S - 1, E, T>(t, b, q);
          float2 x = cscale(v[b * RL + q], a.scale);
          if (arow) x = cadd(x, arow[m]);
          orow[m] = x;
        }
      if (t == 0) orow[N] = make_float2(0.f, 0.f);
    }
  }
}

int set_smem(const void *fn, size_t bytes) { return func_smem(fn, bytes); }

int line_plan_create(int n, LinePlan *p) {
  if (!radix_list(n, &p->rl)) return CRAVA_GPU_ERR_ARG;
  std::vector<float2> tw(n);
  for (int k = 0; k < n; ++k) {
    double ang = -2.0 * M_PI * (double)k / (double)n;
    tw[k] = make_float2((float)cos(ang), (float)sin(ang));
  }
  CRAVA_CUDA_TRY(cudaMalloc(&p->tw, sizeof(float2) * n));
  CRAVA_CUDA_TRY(cudaMemcpy(p->tw, tw.data(), sizeof(float2) * n, cudaMemcpyHostToDevice));
  return CRAVA_GPU_OK;
}

}  // namespace

bool radix_list(int n, RadixList *out) {
  out->n = n;
  out->nr = 0;
  if (n < 1) return false;
  int m = n;
  int r[16];
  int nr = 0;
  // radix 8 while possible, then 4, then 2; then the odd primes.
  const int order[6] = {8, 4, 2, 3, 5, 7};
  for (int i = 0; i < 6; ++i)
    while (m % order[i] == 0) {
      if (nr >= 16) return false;
      r[nr++] = order[i];
      m /= order[i];
    }
  if (m != 1) return false;
  int Ns = 1;
  for (int s = 0; s < nr; ++s) {
    Stage &st = out->st[s];
    st.R = r[s];
    st.Ns = Ns;
    st.m = n / r[s];
    st.tstep = n / (Ns * r[s]);
    st.fNs = make_fastdiv((uint32_t)Ns);
    st.fm = make_fastdiv((uint32_t)st.m);
    Ns *= r[s];
  }
  out->nr = nr;
  return true;
}

float forward_scale(const Geom &g, int type) {
  if (type == CRAVA_GRID_COVARIANCE) return 1.0f;
  return 1.0f / sqrtf((float)(g.nxp * g.nyp * g.nzp));
}
float inverse_scale(const Geom &g, int type) {
  if (type == CRAVA_GRID_COVARIANCE) return (float)(1.0 / ((double)g.nxp * g.nyp * g.nzp));
  return (float)(1.0 / sqrt((float)(g.nxp * g.nyp * g.nzp)));
}

int fft_plans_create(const Geom &g, FftPlans *p) {
  p->g = g;
  p->x_even = (g.nxp % 2) == 0;
  int rc;
  if ((rc = line_plan_create(p->x_even ? g.nxp / 2 : g.nxp, &p->x))) return rc;
  if ((rc = line_plan_create(g.nyp, &p->y))) return rc;
  if ((rc = line_plan_create(g.nzp, &p->z))) return rc;
  if (p->x_even) {
    int h = g.nxp / 2;
    std::vector<float2> post(h + 1);
    for (int k = 0; k <= h; ++k) {
      double ang = -2.0 * M_PI * (double)k / (double)g.nxp;
      post[k] = make_float2((float)cos(ang), (float)sin(ang));
    }
    CRAVA_CUDA_TRY(cudaMalloc(&p->xpost, sizeof(float2) * (h + 1)));
    CRAVA_CUDA_TRY(cudaMemcpy(p->xpost, post.data(), sizeof(float2) * (h + 1), cudaMemcpyHostToDevice));
  }
  return plane_xy_tables(g, &p->twq, &p->twy);
}

void fft_plans_destroy(FftPlans *p) {
  cudaFree(p->x.tw); cudaFree(p->y.tw); cudaFree(p->z.tw); cudaFree(p->xpost);
  cudaFree(p->twq); cudaFree(p->twy);
  p->x.tw = p->y.tw = p->z.tw = p->xpost = p->twq = p->twy = nullptr;
}

int fft_rows(const FftPlans &p, float *grid, int dir, float scale, cudaStream_t s,
             const float *addend, const float *src) {
  RowArgs a;
  a.addend = addend;
  a.src = src ? src : grid;
  a.grid = grid;
  a.nrows = (long long)p.g.nyp * p.g.nzp;
  a.rnxp = p.g.rnxp;
  a.nxp = p.g.nxp;
  a.rl = p.x.rl;
  a.tw = p.x.tw;
  a.post = p.xpost;
  a.scale = scale;
  const int n = a.rl.n;
  if (p.x_even && p.rows_x != 0 && rr::supported(n)) {
#define CRAVA_ROWS_RR(NN)                                                                      \
    if (n == NN) {                                                                             \
      const dim3 g2((unsigned)((a.nrows + RrRows<NN>::ROWS - 1) / RrRows<NN>::ROWS));          \
      const size_t sm2 = sizeof(float2) * ((size_t)rr::tw_slots<NN>() + NN + 1 + (size_t)RrRows<NN>::ROWS * RrRows<NN>::P); \
      const void *f = dir < 0 ? (const void *)k_rows_rr<NN, -1> : (const void *)k_rows_rr<NN, 1>; \
      int r2 = set_smem(f, sm2);                                                               \
      if (r2) return r2;                                                                       \
      if (dir < 0) k_rows_rr<NN, -1><<<g2, RrRows<NN>::NTH, sm2, s>>>(a);                      \
      else k_rows_rr<NN, 1><<<g2, RrRows<NN>::NTH, sm2, s>>>(a);                               \
      CRAVA_LAUNCH_CHECK();                                                                    \
      return CRAVA_GPU_OK;                                                                     \
    }
    CRAVA_ROWS_RR(64) CRAVA_ROWS_RR(128) CRAVA_ROWS_RR(256) CRAVA_ROWS_RR(512)
#undef CRAVA_ROWS_RR
  }
  if (p.x_even) {
    const size_t sm2 = sizeof(float2) * (n + n + 1 + (size_t)n * (kRR + 1));
    const dim3 g2((unsigned)((a.nrows + kRR - 1) / kRR));
#define CRAVA_ROWS_IP(NN)                                                                    \
    if (n == NN) {                                                                           \
      const void *f = dir < 0 ? (const void *)k_rows_ip<NN, -1> : (const void *)k_rows_ip<NN, 1>; \
      int r2 = set_smem(f, sm2);                                                             \
      if (r2) return r2;                                                                     \
      if (dir < 0) k_rows_ip<NN, -1><<<g2, kThreads, sm2, s>>>(a);                           \
      else k_rows_ip<NN, 1><<<g2, kThreads, sm2, s>>>(a);                                    \
      CRAVA_LAUNCH_CHECK();                                                                  \
      return CRAVA_GPU_OK;                                                                   \
    }
    CRAVA_ROWS_IP(32) CRAVA_ROWS_IP(48) CRAVA_ROWS_IP(64) CRAVA_ROWS_IP(96) CRAVA_ROWS_IP(128)
    CRAVA_ROWS_IP(256)
#undef CRAVA_ROWS_IP
  }
  size_t smem = sizeof(float2) * (n + (p.x_even ? n + 1 : 0) + 2 * kRows * (n + 1));
  dim3 grd((unsigned)((a.nrows + kRows - 1) / kRows));
  const void *fn;
  if (dir < 0) fn = p.x_even ? (const void *)k_rows<-1, true> : (const void *)k_rows<-1, false>;
  else fn = p.x_even ? (const void *)k_rows<1, true> : (const void *)k_rows<1, false>;
  int rc = set_smem(fn, smem);
  if (rc) return rc;
  if (dir < 0) {
    if (p.x_even) k_rows<-1, true><<<grd, kThreads, smem, s>>>(a);
    else k_rows<-1, false><<<grd, kThreads, smem, s>>>(a);
  } else {
    if (p.x_even) k_rows<1, true><<<grd, kThreads, smem, s>>>(a);
    else k_rows<1, false><<<grd, kThreads, smem, s>>>(a);
  }
  CRAVA_LAUNCH_CHECK();
  return CRAVA_GPU_OK;
}

// Column tile width of the in-place column pass (0 selects the ping-pong
// pass); CRAVA_COLS_TX=0|8|16 overrides the default for measurements.
static int cols_tile_width(int n) {
  static int tx = -1;
  if (tx < 0) {
    const char *e = getenv("CRAVA_COLS_TX");
    tx = e ? atoi(e) : -2;
    if (tx != 0 && tx != 8 && tx != 16) tx = -2;
  }
  if (tx != -2) return tx;
  return n <= 256 ? 16 : 8;  // measured best on B200 at 256x256x512
}

static int cols(const LinePlan &lp, float2 *data, int ninner, long long es,
                long long outer_stride, int nouter, int dir, float scale, int tile, cudaStream_t s,
                const ZPrior *zp = nullptr) {
  ColArgs a;
  a.data = data;
  a.ninner = ninner;
  a.elem_stride = es;
  a.outer_stride = outer_stride;
  a.rl = lp.rl;
  a.tw = lp.tw;
  a.scale = scale;
  const int n = lp.rl.n;
  size_t smem = sizeof(float2) * (n + 2 * kColTile * n);
  dim3 grd((ninner + kColTile - 1) / kColTile, nouter);
  if ((tile == 1 || tile < 0) && rr::supported(n) && scale == 1.0f) {
    // register-resident pass over the ninner * nouter lines taken flat:
    // line f = i + ninner o starts at i + outer_stride o
    ColRRArgs r;
    r.data = data;
    r.nlines = (long long)ninner * nouter;
    r.A = (uint32_t)ninner;
    r.fa = make_fastdiv((uint32_t)ninner);
    r.B = outer_stride;
    r.es = es;
    r.tw = lp.tw;
    if (zp && dir < 0) r.zp = *zp;
    if (r.nlines >= (1LL << 31)) return CRAVA_GPU_ERR_ARG;
    const bool flat = outer_stride == ninner;
    // 16-byte accesses need the two lines of a thread adjacent and aligned:
    // lengths whose threads hold two lines (CPT 2), flat lines, even stride
    const bool two = (n == 64 || n == 512);  // RrCols<n>::CPT == 2
    const bool vec = two && flat && (es % 2 == 0) && (reinterpret_cast<uintptr_t>(data) % 16 == 0);
    const dim3 g2((unsigned)((r.nlines + kRrTX - 1) / kRrTX));
#define CRAVA_COLS_RR(NN)                                                                           \
    if (n == NN) {                                                                                  \
      const size_t sm2 = sizeof(float2) * ((size_t)NN + (size_t)NN * kRrTX);                        \
      const void *f = dir < 0 ? (vec ? (const void *)k_cols_rr<NN, -1, true> : (const void *)k_cols_rr<NN, -1, false>) \
                              : (vec ? (const void *)k_cols_rr<NN, 1, true> : (const void *)k_cols_rr<NN, 1, false>);  \
      int r2 = set_smem(f, sm2);                                                                    \
      if (r2) return r2;                                                                            \
      constexpr int nth = RrCols<NN>::NTH;                                                          \
      if (dir < 0) {                                                                                \
        if (vec) k_cols_rr<NN, -1, true><<<g2, nth, sm2, s>>>(r);                                   \
        else k_cols_rr<NN, -1, false><<<g2, nth, sm2, s>>>(r);                                      \
      } else {                                                                                      \
        if (vec) k_cols_rr<NN, 1, true><<<g2, nth, sm2, s>>>(r);                                    \
        else k_cols_rr<NN, 1, false><<<g2, nth, sm2, s>>>(r);                                       \
      }                                                                                             \
      CRAVA_LAUNCH_CHECK();                                                                         \
      return CRAVA_GPU_OK;                                                                          \
    }
    CRAVA_COLS_RR(64) CRAVA_COLS_RR(128) CRAVA_COLS_RR(256) CRAVA_COLS_RR(512)
#undef CRAVA_COLS_RR
  }
  const int tx = tile > 1 || tile == 0 ? tile : cols_tile_width(n);
#define CRAVA_COLS_CT(NN)                                                                   \
  if (n == NN && tx > 0) {                                                                  \
    const dim3 g2((ninner + tx - 1) / tx, nouter);                                          \
    const size_t sm2 = sizeof(float2) * (NN + (size_t)cols_pitch(tx) *                      \
                                         padded_rows(NN, cols_padr(NN, tx)));               \
    const void *f = tx == 16 ? (dir < 0 ? (const void *)k_cols_ip<NN, -1, 16> : (const void *)k_cols_ip<NN, 1, 16>) \
                             : (dir < 0 ? (const void *)k_cols_ip<NN, -1, 8> : (const void *)k_cols_ip<NN, 1, 8>);  \
    int r2 = set_smem(f, sm2);                                                              \
    if (r2) return r2;                                                                      \
    if (tx == 16) {                                                                         \
      if (dir < 0) k_cols_ip<NN, -1, 16><<<g2, kThreads, sm2, s>>>(a);                      \
      else k_cols_ip<NN, 1, 16><<<g2, kThreads, sm2, s>>>(a);                               \
    } else {                                                                                \
      if (dir < 0) k_cols_ip<NN, -1, 8><<<g2, kThreads, sm2, s>>>(a);                       \
      else k_cols_ip<NN, 1, 8><<<g2, kThreads, sm2, s>>>(a);                                \
    }                                                                                       \
    CRAVA_LAUNCH_CHECK();                                                                   \
    return CRAVA_GPU_OK;                                                                    \
  }                                                                                         \
  if (n == NN) {                                                                            \
    const void *f = dir < 0 ? (const void *)k_cols_ct<NN, -1> : (const void *)k_cols_ct<NN, 1>; \
    int r2 = set_smem(f, smem);                                                             \
    if (r2) return r2;                                                                      \
    if (dir < 0) k_cols_ct<NN, -1><<<grd, kThreads, smem, s>>>(a);                          \
    else k_cols_ct<NN, 1><<<grd, kThreads, smem, s>>>(a);                                   \
    CRAVA_LAUNCH_CHECK();                                                                   \
    return CRAVA_GPU_OK;                                                                    \
  }
  CRAVA_COLS_CT(64) CRAVA_COLS_CT(128) CRAVA_COLS_CT(256) CRAVA_COLS_CT(512)
  CRAVA_COLS_CT(96) CRAVA_COLS_CT(160) CRAVA_COLS_CT(192) CRAVA_COLS_CT(200) CRAVA_COLS_CT(300)
  CRAVA_COLS_CT(384)
#undef CRAVA_COLS_CT
  const void *fn = dir < 0 ? (const void *)k_cols<-1> : (const void *)k_cols<1>;
  int rc = set_smem(fn, smem);
  if (rc) return rc;
  if (dir < 0) k_cols<-1><<<grd, kThreads, smem, s>>>(a);
  else k_cols<1><<<grd, kThreads, smem, s>>>(a);
  CRAVA_LAUNCH_CHECK();
  return CRAVA_GPU_OK;
}

bool cols_tunable(int n) {
  for (int m : {64, 128, 256, 512, 96, 160, 192, 200, 300, 384})
    if (n == m) return true;
  return false;
}

bool cols_rr(int n) { return rr::supported(n); }
static_assert(RrCols<64>::CPT == 2 && RrCols<512>::CPT == 2 && RrCols<128>::CPT == 1 && RrCols<256>::CPT == 1,
              "the 16-byte path of k_cols_rr is chosen for the lengths whose threads hold two lines");

int fft_cols_y(const FftPlans &p, float2 *grid, int dir, cudaStream_t s) {
  const Geom &g = p.g;
  return cols(p.y, grid, g.cnxp, g.cnxp, (long long)g.cnxp * g.nyp, g.nzp, dir, 1.0f, p.tile_y == 2 ? -1 : p.tile_y, s);
}

bool z_prior_supported(const FftPlans &p) {
  // the register-resident pass (tile -1 / 1) or its TMA-fed form (2); the
  // TMA pass falls back to the register-resident one where a grid does not
  // allow it, which applies the rule too
  return rr::supported(p.g.nzp) && (p.tile_z == -1 || p.tile_z == 1 || p.tile_z == 2);
}

int fft_cols_z(const FftPlans &p, float2 *grid, int dir, cudaStream_t s, const ZPrior *zp) {
  const Geom &g = p.g;
  if (zp && zp->inv && !z_prior_supported(p)) return CRAVA_GPU_ERR_ARG;
  // the TMA-fed pass (tile choice 2): faster alone; in the unit's lane
  // overlap it pays beside the fused x + y pass (5.23 against 5.85 ms per
  // 256x256x512x5 unit) and not beside the separate passes (5.92 against
  // 5.40 ms), so it is built in where the fused pass is
  const bool tma = p.tile_z == 2 || (p.tile_z == -1 && use_plane_xy(p));
  if (tma && cols_z_tma_supported(g, grid)) return cols_z_tma(p, grid, dir, s, zp);
  return cols(p.z, grid, g.cnxp, (long long)g.cnxp * g.nyp, g.cnxp, g.nyp, dir, 1.0f, p.tile_z == 2 ? -1 : p.tile_z, s,
              zp);
}

int fft3d_r2c(const FftPlans &p, float *grid, int type, cudaStream_t s) {
  int rc;
  if (use_plane_xy(p)) {
    if ((rc = plane_xy(p, grid, grid, -1, forward_scale(p.g, type), nullptr, s))) return rc;
    return fft_cols_z(p, reinterpret_cast<float2 *>(grid), -1, s);
  }
  if ((rc = fft_rows(p, grid, -1, forward_scale(p.g, type), s))) return rc;
  if ((rc = fft_cols_y(p, reinterpret_cast<float2 *>(grid), -1, s))) return rc;
  return fft_cols_z(p, reinterpret_cast<float2 *>(grid), -1, s);
}

int fft3d_c2r(const FftPlans &p, float *grid, int type, cudaStream_t s, const float *addend) {
  int rc;
  if ((rc = fft_cols_z(p, reinterpret_cast<float2 *>(grid), 1, s))) return rc;
  if (use_plane_xy(p)) return plane_xy(p, grid, grid, 1, inverse_scale(p.g, type), addend, s);
  if ((rc = fft_cols_y(p, reinterpret_cast<float2 *>(grid), 1, s))) return rc;
  return fft_rows(p, grid, 1, inverse_scale(p.g, type), s, addend);
}

}  // namespace crava
