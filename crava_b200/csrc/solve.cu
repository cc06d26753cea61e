// solve.cu -- per-kz operator tables and the per-(kx,ky,kz) posterior solve.
//
// Replaces the hot loop of Crava::computePostMeanResidAndFFTCov
// (src/crava.cpp:1042-1151) with SeismicParametersHolder::
// getNextParameterCovariance (src/seismicparametersholder.cpp:355-427) and
// Crava::getNextErrorVariance (src/crava.cpp:1297-1334).  One thread owns
// one complex bin; all matrices stay in registers.
//
// Structure used (constant thickness, src/crava.cpp:1046-1058):
//   K = diag(wd) A, wd_l(k) = D(k) conj(W_l(k)), A real ntheta x 3,
//   S real symmetric 3x3 (|Re| of the prior spectra times Sigma0),
// so  K S K^H = diag(wd) (A S A^T) diag(wd)^H and K S = diag(wd) (A S):
//   B = A S A^T (real), M_lm = wd_l conj(wd_m) B_lm + Sigma_e,lm,
//   L L^H = M,  X = M^-1 K S,  S_post = S - (KS)^H X,
//   mu_post = mu + X^H (d - K mu),  r = d - K mu_post.
// Band gating and the prior fallback on a failed factorisation follow the
// reference (src/crava.cpp:1098, 1109-1111): outside the band, or when
// M00 <= 0 or a pivot of M/M00 is <= 1e-20 (libs/lib/lib_matr.c:20,
// 103-105, 114, 145), the bin keeps mu, S and r = d.
#include <math.h>
#include <stdlib.h>

#include <algorithm>

#include <vector>

#include "fft_core.cuh"
#include "solve.cuh"
#include "solve_bin.cuh"
#include "woodbury.cuh"

namespace crava {

namespace {

constexpr int kThreads = 256;
using sb::tri;

// ------------------------------------------------------------------ tables
__global__ void k_kz_tables(const float *__restrict__ wav,
                            const float *__restrict__ wnorm_in, int has_norm,
                            int nzp, int nt, int nz, double lz, double mrt,
                            float low_cut, float high_cut, int mode, KzTables t) {
  extern __shared__ double shd[];
  const int l = blockIdx.x, tid = threadIdx.x, nth = blockDim.x;
  const int cnzp = nzp / 2 + 1;
  double *cs = shd;               // cos(2 pi m / nzp)
  double *sn = cs + nzp;          // sin(2 pi m / nzp)
  double *red = sn + nzp;         // 2 * nth partial sums
  float2 *W = reinterpret_cast<float2 *>(red + 2 * nth);
  float2 *G = W + cnzp;
  float *w = reinterpret_cast<float *>(G + cnzp);
  float *e = w + nzp, *f = e + nzp, *g = f + nzp;
  const float *wl = wav + (long long)l * nzp;
  for (int m = tid; m < nzp; m += nth) {
    double s, c;
    sincospi(2.0 * m / nzp, &s, &c);
    cs[m] = c; sn[m] = s;
    w[m] = wl[m];
  }
  __syncthreads();
  // Wavelet1D difference constructors (src/wavelet1D.cpp:420-479):
  // forward, backward, then central difference, cyclic.
  for (int i = tid; i < nzp; i += nth) e[i] = (i == nzp - 1) ? w[0] - w[i] : w[i + 1] - w[i];
  __syncthreads();
  for (int i = tid; i < nzp; i += nth) f[i] = (i == 0) ? e[0] - e[nzp - 1] : e[i] - e[i - 1];
  __syncthreads();
  for (int i = tid; i < nzp; i += nth) {
    float d = (i == 0) ? f[1] - f[nzp - 1] : (i == nzp - 1) ? f[0] - f[i - 1] : f[i + 1] - f[i - 1];
    g[i] = (float)(0.5 * (double)d);
  }
  // Wavelet::findNorm (src/wavelet.cpp:789-808): time-domain L2 norms.
  double sw = 0.0, sg = 0.0;
  __syncthreads();
  for (int i = tid; i < nzp; i += nth) {
    sw += (double)(w[i] * w[i]);
    sg += (double)(g[i] * g[i]);
  }
  red[tid] = sw; red[nth + tid] = sg;
  __syncthreads();
  for (int off = nth / 2; off > 0; off >>= 1) {
    if (tid < off) { red[tid] += red[tid + off]; red[nth + tid] += red[nth + tid + off]; }
    __syncthreads();
  }
  const float wn = has_norm ? wnorm_in[l] : (float)sqrt(red[0]);
  const float gn = (float)sqrt(red[nth]);
  // Unnormalised forward spectra (Wavelet::fft1DInPlace), in double.
  for (int k = tid; k < cnzp; k += nth) {
    double wr = 0, wi = 0, gr = 0, gi = 0;
    for (int n = 0; n < nzp; ++n) {
      int m = (int)(((long long)k * n) % nzp);
      double c = cs[m], s = -sn[m];
      wr += w[n] * c; wi += w[n] * s;
      gr += g[n] * c; gi += g[n] * s;
    }
    W[k] = make_float2((float)wr, (float)wi);
    G[k] = make_float2((float)gr, (float)gi);
  }
  __syncthreads();
  for (int k = tid; k < nzp; k += nth) {
    // Wavelet::getCAmp(k): Hermitian mirror for k >= nzp/2+1 (src/wavelet.cpp:308-324)
    float2 ca = k < cnzp ? W[k] : make_float2(W[nzp - k].x, -W[nzp - k].y);
    float2 cg = k < cnzp ? G[k] : make_float2(G[nzp - k].x, -G[nzp - k].y);
    // diff1Operator: FFT of [-1, 0, ..., 0, 1] = -1 + e^{2 pi i k/nzp}
    float2 kD = make_float2((float)(cs[k] - 1.0), (float)sn[k]);
    const long long o = (long long)k * nt + l;
    if (mode == 1) {
      // non-constant thickness (src/crava.cpp:1059-1083): K = diag(D) A,
      // errMult1 = 1/|W|, errMult2 = D3/|E3| with D3 the spectrum of the
      // central difference of the backward difference of the difference
      // operator (:938-940), here i (sin 2t - 2 sin t), t = 2 pi k / nzp;
      // errMult3 = fillInverseAbskWRobust (:1358-1384)
      t.wd[o] = kD;
      t.e1[o] = make_float2(1.0f / wn, 0.0f);
      const double s1 = sn[k], s2 = sn[(int)((2LL * k) % nzp)];
      const float m2 = 1.0f / gn;
      t.e2[o] = make_float2(0.0f * m2, (float)(s2 - 2.0 * s1) * m2);
      // getCAmp(k, 0.999): the spectrum of the slightly stretched wavelet
      const int refk = k < cnzp ? k : nzp - k;
      const float scale = 0.999f;
      const float omega = __fdiv_rn((float)refk, scale);
      float2 vf = make_float2(0.0f, 0.0f);
      if (omega < (float)cnzp) {
        const int omL = (int)floorf(omega);
        int omU = omL + 1;
        if (omU >= cnzp) omU -= 1;
        const float dO = __fsub_rn(omega, (float)omL), dL = __fsub_rn(1.0f, dO);
        vf.x = __fadd_rn(__fmul_rn(W[omL].x, dL), __fmul_rn(W[omU].x, dO));
        vf.y = __fadd_rn(__fmul_rn(W[omL].y, dL), __fmul_rn(W[omU].y, dO));
        if (k >= cnzp) vf.y = -vf.y;
      }
      vf.x = __fdiv_rn(vf.x, scale);
      vf.y = __fdiv_rn(vf.y, scale);
      const float mod = __fadd_rn(__fmul_rn(ca.x, ca.x), __fmul_rn(ca.y, ca.y));
      const float modF = __fadd_rn(__fmul_rn(vf.x, vf.x), __fmul_rn(vf.y, vf.y));
      const float maxMod = fmaxf(mod, modF);
      // float(1.0 / sqrt(maxMod)): the float square root, a double quotient
      t.e3[o] = maxMod > 0.0f ? (float)(1.0 / (double)__fsqrt_rn(maxMod)) : wn * nzp * nzp * 100.0f;
    } else {
      float2 kw = make_float2(ca.x, -ca.y);  // fillkW (src/crava.cpp:1336-1344)
      t.wd[o] = make_float2(kD.x * kw.x - kD.y * kw.y, kD.x * kw.y + kD.y * kw.x);
      t.e1[o] = make_float2(ca.x / wn, -(ca.y / wn));  // fillkWNorm (:1346-1355)
      t.e2[o] = make_float2(cg.x / gn, -(cg.y / gn));
      t.e3[o] = 1.0f;
    }
    if (l == 0) {
      int mk = k < nzp - k ? k : nzp - k;
      float rf = (float)((nz * 1000.0f) / (lz * nzp) * mk);  // src/crava.cpp:1044
      t.inv[k] = (rf > low_cut * mrt) && (rf < high_cut);
    }
  }
}

struct SolveArgs {
  SolveConsts c;
  SolveGrids g;
  KzTables t;
  long long csize, plane;
  long long bpp;  // blocks per kz plane
  long long nslots = 0;  // kz planes visited (t.order[0 .. nslots))
  DevCounters *counters;
  // Woodbury form: the per-plane tables and the list of the blocks it
  // defers to the square-root kernel
  const sb::WbTable *wb = nullptr;
  int *list = nullptr;  // deferred blocks (count in counters->deferred)
};

// Square-root form (solve_bin.cuh): the FP64 and mixed forms.  One kz
// plane per CTA: the CTA first stages the plane's per-kz constants of M in
// shared memory.  The factor lives either in shared memory, one entry
// column per thread (LREG false), or in registers (LREG true); the first
// two columns of Y = L^-1 K S (and, mixed form, the FP64 prior-mean
// residual used by the refinement step) are in shared memory.  A factor in
// shared memory costs about 180 16-byte accesses per inverted bin at five
// angles, which bounds that shape by the SM's shared-memory bandwidth; in
// registers it costs occupancy instead.
template <int NT, int PREC, int NTH, bool LREG>
struct SqSmem {
  static constexpr int NP = NT * (NT + 1) / 2;
  static constexpr size_t kconst = (sizeof(sb::KzConst<NT>) + 15) / 16 * 16;
  static constexpr size_t per_thread =
      PREC == 0 ? sizeof(double2) * ((LREG ? 0 : NP) + 2 * NT)
                : sizeof(double2) * NT + sizeof(float2) * ((LREG ? 0 : NP) + 2 * NT);
  static constexpr size_t bytes = kconst + per_thread * NTH;
};

// One block's bins (block blk of the solve's grid); every thread reaches
// the one barrier, after which threads without a bin return.
template <int NT, int PREC, int NTH, bool LREG>
__device__ __forceinline__ void sq_block(const SolveArgs &a, long long blk) {
  using SM = SqSmem<NT, PREC, NTH, LREG>;
  extern __shared__ double2 sq_sm[];
  auto &kc = *reinterpret_cast<sb::KzConst<NT> *>(sq_sm);
  char *area = reinterpret_cast<char *>(sq_sm) + SM::kconst;
  const int slot = (int)(blk / a.bpp);
  const long long off = (long long)(blk % a.bpp) * NTH + threadIdx.x;
  const int k = a.t.order ? a.t.order[slot] : slot;
  const bool inv = a.t.inv[k] != 0;
  const long long o = (long long)k * NT;
  if (inv) sb::kz_const_fill<NT>(kc, a.c, a.t.wd + o, a.t.e1 + o, a.t.e2 + o, a.t.e3 + o, threadIdx.x);
  __syncthreads();
  if (off >= a.plane) return;
  const long long idx = (long long)k * a.plane + off;
  float2 c6[6];
#pragma unroll
  for (int t = 0; t < 6; ++t) c6[t] = a.g.cov[t][idx];
  if (!inv) {
    sb::prior_only<PREC>(a.c, c6);
    bool nonfinite = false;
#pragma unroll
    for (int t = 0; t < 6; ++t) { a.g.cov[t][idx] = c6[t]; nonfinite |= !sb::fin2(c6[t]); }
    if (a.counters) sb::count(a.counters, false, nonfinite);
    return;
  }
  const sb::Sym3d S = sb::prior_exact(c6, a.c.var0);
  const float2 ec = a.g.err[idx];
  const sb::GlobalIn gin{&a.g, idx};
  bool solved, fin = true, refined = false;
  if (PREC == 0) {
    double2 *base = reinterpret_cast<double2 *>(area) + threadIdx.x;
    if (LREG) {
      double2 L[SM::NP];
      const sb::SmemTri<double2, NTH> Y{base};
      solved = sb::solve_bin_fp64_sq<NT>(&L[0], Y, a.c, kc, S, fabs((double)ec.x), a.g, idx, gin, &fin);
    } else {
      const sb::SmemTri<double2, NTH> L{base};
      const sb::SmemTri<double2, NTH> Y{base + NTH * SM::NP};
      solved = sb::solve_bin_fp64_sq<NT>(L, Y, a.c, kc, S, fabs((double)ec.x), a.g, idx, gin, &fin);
    }
  } else {
    double2 *vbase = reinterpret_cast<double2 *>(area) + threadIdx.x;
    float2 *fbase = reinterpret_cast<float2 *>(reinterpret_cast<double2 *>(area) + NTH * NT) + threadIdx.x;
    const sb::SmemTri<double2, NTH> V{vbase};
    if (LREG) {
      float2 Lf[SM::NP];
      const sb::SmemTri<float2, NTH> Yf{fbase};
      solved = sb::solve_bin_mixed_sq<NT>(&Lf[0], Yf, V, a.c, kc, S, a.c.kappa_refine, fabsf(ec.x),
                                          fabs((double)ec.x), a.g, idx, gin, &fin, &refined);
    } else {
      const sb::SmemTri<float2, NTH> Lf{fbase};
      const sb::SmemTri<float2, NTH> Yf{fbase + NTH * SM::NP};
      solved = sb::solve_bin_mixed_sq<NT>(Lf, Yf, V, a.c, kc, S, a.c.kappa_refine, fabsf(ec.x),
                                          fabs((double)ec.x), a.g, idx, gin, &fin, &refined);
    }
  }
  if (!solved) {
    // the reference keeps the prior (src/crava.cpp:1109-1111): the mean and
    // the data stay, the covariance takes the prior of this form's
    // arithmetic (FP64: the double prior rounded; mixed: the float prior)
    sb::prior_only<PREC>(a.c, c6);
#pragma unroll
    for (int t = 0; t < 6; ++t) { a.g.cov[t][idx] = c6[t]; fin &= sb::fin2(c6[t]); }
#pragma unroll
    for (int q = 0; q < 3; ++q) fin &= sb::fin2(a.g.mu[q][idx]);
#pragma unroll
    for (int l = 0; l < NT; ++l) fin &= sb::fin2(a.g.data[l][idx]);
  }
  if (a.counters) {
    sb::count(a.counters, !solved, !fin);
    if (PREC == 1) {
      const unsigned m = __activemask();
      const unsigned br = __ballot_sync(m, refined);
      if (br && (threadIdx.x & 31) == __ffs(m) - 1) atomicAdd(&a.counters->refined, (unsigned long long)__popc(br));
    }
  }
}

template <int NT, int PREC, int NTH, int MINB, bool LREG>
__global__ void __launch_bounds__(NTH, MINB) k_solve_sq(SolveArgs a) {
  sq_block<NT, PREC, NTH, LREG>(a, blockIdx.x);
}

// The blocks the Woodbury kernel deferred (a.list, a.counters->deferred of
// them), walked by a small fixed grid: with no deferred block it costs one
// counter read per CTA.
template <int NT, int NTH, int MINB>
__global__ void __launch_bounds__(NTH, MINB) k_solve_sq_list(SolveArgs a) {
  const unsigned long long n = *(volatile unsigned long long *)&a.counters->deferred;
  for (unsigned long long i = blockIdx.x; i < n; i += gridDim.x) {
    __syncthreads();  // the previous block's per-kz constants are no longer read
    sq_block<NT, 0, NTH, true>(a, a.list[i]);
  }
}

// The square-root solve with the bin inputs staged ahead of the compute.
// Each thread runs BPT bins of its kz plane in turn; while bin j computes,
// the 10 + NT input spectra of bin j + 1 travel by cp.async into the
// thread's own slot of a two-deep staging buffer in shared memory (a
// band-gated plane stages only its six covariance spectra), and the bin's
// inputs are read from there (the end-of-bin re-reads included) instead of
// from global memory: the loads that stalled the one-bin-per-thread kernel
// overlap the FP64 work of the previous bin.  Only the thread that staged a
// slot reads it, so no block barrier is needed between bins.  The factor is
// in registers; the first two columns of Y (FP64 form) or the FP64
// prior-mean residual and two FP32 columns of Y (mixed form) are in shared
// memory.
template <int NT, int PREC, int NTH>
struct PfSmem {
  static constexpr int NIN = 10 + NT;
  static constexpr size_t kconst = (sizeof(sb::KzConst<NT>) + 15) / 16 * 16;
  static constexpr size_t scratch =
      PREC == 0 ? sizeof(double2) * 2 * NT : sizeof(double2) * NT + sizeof(float2) * 2 * NT;
  static constexpr size_t bytes = kconst + (scratch + sizeof(float2) * 2 * NIN) * NTH;
};

template <int NT, int PREC, int NTH, int MINB, int BPT>
__global__ void __launch_bounds__(NTH, MINB) k_solve_pf(SolveArgs a) {
  using SM = PfSmem<NT, PREC, NTH>;
  constexpr int NIN = SM::NIN;
  extern __shared__ double2 pf_sm[];
  auto &kc = *reinterpret_cast<sb::KzConst<NT> *>(pf_sm);
  char *area = reinterpret_cast<char *>(pf_sm) + SM::kconst;
  double2 *dscr = reinterpret_cast<double2 *>(area) + threadIdx.x;
  float2 *stage = reinterpret_cast<float2 *>(area + SM::scratch * NTH) + threadIdx.x;  // [2][NIN][NTH]
  const int slot = (int)(blockIdx.x / a.bpp);
  const long long base = (long long)(blockIdx.x % a.bpp) * NTH * BPT;
  const int k = a.t.order ? a.t.order[slot] : slot;
  const bool inv = a.t.inv[k] != 0;
  const long long o = (long long)k * NT;
  const long long pbase = (long long)k * a.plane;
  if (inv) sb::kz_const_fill<NT>(kc, a.c, a.t.wd + o, a.t.e1 + o, a.t.e2 + o, a.t.e3 + o, threadIdx.x);

  auto issue = [&](int j) {
    const long long off = base + (long long)j * NTH + threadIdx.x;
    if (off < a.plane) {
      const long long idx = pbase + off;
      float2 *dst = stage + (j & 1) * NIN * NTH;
      if (inv) {
#pragma unroll
        for (int q = 0; q < 3; ++q) cp_async8(dst + q * NTH, a.g.mu[q] + idx);
#pragma unroll
        for (int l = 0; l < NT; ++l) cp_async8(dst + (3 + l) * NTH, a.g.data[l] + idx);
        cp_async8(dst + (9 + NT) * NTH, a.g.err + idx);
      }
#pragma unroll
      for (int t = 0; t < 6; ++t) cp_async8(dst + (3 + NT + t) * NTH, a.g.cov[t] + idx);
    }
    cp_async_commit();
  };
  issue(0);
  __syncthreads();  // the per-kz constants
  for (int j = 0; j < BPT; ++j) {
    if (j + 1 < BPT) issue(j + 1);
    else cp_async_commit();  // an empty group keeps the wait count uniform
    cp_async_wait<1>();      // bin j has landed in its slot
    const long long off = base + (long long)j * NTH + threadIdx.x;
    if (off >= a.plane) continue;
    const long long idx = pbase + off;
    const sb::StagedIn<NT, NTH> in{stage + (j & 1) * NIN * NTH};
    float2 c6[6];
#pragma unroll
    for (int t = 0; t < 6; ++t) c6[t] = in.cov(t);
    if (!inv) {
      sb::prior_only<PREC>(a.c, c6);
      bool nonfinite = false;
#pragma unroll
      for (int t = 0; t < 6; ++t) { a.g.cov[t][idx] = c6[t]; nonfinite |= !sb::fin2(c6[t]); }
      if (a.counters) sb::count(a.counters, false, nonfinite);
      continue;
    }
    const sb::Sym3d S = sb::prior_exact(c6, a.c.var0);
    const float2 ec = in.err();
    bool solved, fin = true, refined = false;
    if (PREC == 0) {
      double2 L[NT * (NT + 1) / 2];
      const sb::SmemTri<double2, NTH> Y{dscr};
      solved = sb::solve_bin_fp64_sq<NT>(&L[0], Y, a.c, kc, S, fabs((double)ec.x), a.g, idx, in, &fin);
    } else {
      float2 Lf[NT * (NT + 1) / 2];
      const sb::SmemTri<double2, NTH> V{dscr};
      const sb::SmemTri<float2, NTH> Yf{reinterpret_cast<float2 *>(reinterpret_cast<double2 *>(area) + NTH * NT) +
                                        threadIdx.x};
      solved = sb::solve_bin_mixed_sq<NT>(&Lf[0], Yf, V, a.c, kc, S, a.c.kappa_refine, fabsf(ec.x),
                                          fabs((double)ec.x), a.g, idx, in, &fin, &refined);
    }
    if (!solved) {
      // the reference keeps the prior (src/crava.cpp:1109-1111)
      sb::prior_only<PREC>(a.c, c6);
#pragma unroll
      for (int t = 0; t < 6; ++t) { a.g.cov[t][idx] = c6[t]; fin &= sb::fin2(c6[t]); }
#pragma unroll
      for (int q = 0; q < 3; ++q) fin &= sb::fin2(in.mu(q));
#pragma unroll
      for (int l = 0; l < NT; ++l) fin &= sb::fin2(in.d(l));
    }
    if (a.counters) {
      sb::count(a.counters, !solved, !fin);
      if (PREC == 1) {
        const unsigned m = __activemask();
        const unsigned br = __ballot_sync(m, refined);
        if (br && (threadIdx.x & 31) == __ffs(m) - 1)
          atomicAdd(&a.counters->refined, (unsigned long long)__popc(br));
      }
    }
  }
  cp_async_wait<0>();
}

template <int PREC, int NTH, int MINB, int BPT>
int launch_solve_pf(SolveArgs a, int nt, cudaStream_t s) {
  a.bpp = (a.plane + (long long)NTH * BPT - 1) / ((long long)NTH * BPT);
  dim3 grd((unsigned)(a.bpp * a.nslots));
  int rc;
#define CRAVA_PF_CASE(N)                                                                          \
  case N: {                                                                                       \
    const size_t smem = PfSmem<N, PREC, NTH>::bytes;                                              \
    if ((rc = func_smem((const void *)k_solve_pf<N, PREC, NTH, MINB, BPT>, smem))) return rc;     \
    k_solve_pf<N, PREC, NTH, MINB, BPT><<<grd, NTH, smem, s>>>(a);                                \
    break;                                                                                        \
  }
  switch (nt) {
    CRAVA_PF_CASE(1) CRAVA_PF_CASE(2) CRAVA_PF_CASE(3) CRAVA_PF_CASE(4)
    CRAVA_PF_CASE(5) CRAVA_PF_CASE(6) CRAVA_PF_CASE(7) CRAVA_PF_CASE(8)
    default: return CRAVA_GPU_ERR_ARG;
  }
#undef CRAVA_PF_CASE
  CRAVA_LAUNCH_CHECK();
  return CRAVA_GPU_OK;
}

template <int PREC, int NTH, int MINB, bool LREG>
int launch_solve_sq(SolveArgs a, int nt, cudaStream_t s) {
  a.bpp = (a.plane + NTH - 1) / NTH;
  dim3 grd((unsigned)(a.bpp * a.nslots));
  int rc;
#define CRAVA_SQ_CASE(N)                                                                          \
  case N: {                                                                                       \
    const size_t smem = SqSmem<N, PREC, NTH, LREG>::bytes;                                        \
    if ((rc = func_smem((const void *)k_solve_sq<N, PREC, NTH, MINB, LREG>, smem))) return rc;    \
    k_solve_sq<N, PREC, NTH, MINB, LREG><<<grd, NTH, smem, s>>>(a);                               \
    break;                                                                                        \
  }
  switch (nt) {
    CRAVA_SQ_CASE(1) CRAVA_SQ_CASE(2) CRAVA_SQ_CASE(3) CRAVA_SQ_CASE(4)
    CRAVA_SQ_CASE(5) CRAVA_SQ_CASE(6) CRAVA_SQ_CASE(7) CRAVA_SQ_CASE(8)
    default: return CRAVA_GPU_ERR_ARG;
  }
#undef CRAVA_SQ_CASE
  CRAVA_LAUNCH_CHECK();
  return CRAVA_GPU_OK;
}

// FP64 solve in the Woodbury form (woodbury.cuh), one bin per thread and
// one kz plane per block (the grid of k_solve_sq with NTH threads, so the
// square-root kernel can take over a block).  A thread first issues the
// loads of all its bin's inputs, then the block stages the part of its
// plane's table the nt angles use in shared memory (the loads are in
// flight meanwhile).  If any bin of the block cannot use the form (plane
// table not usable, prior not positive definite, lambda m_i + 1 not
// positive), the block writes nothing, appends its index to the deferred
// list, and k_solve_sq_list solves it in the square-root form.  Band-gated
// blocks write the prior covariance as k_solve_sq does.
template <int NT>
struct RegIn {  // a bin's inputs held in registers
  float2 m[3], d[NT];
};
template <int NT>
struct RegInAcc {
  const RegIn<NT> *r;
  __device__ __forceinline__ float2 mu(int q) const { return r->m[q]; }
  __device__ __forceinline__ float2 d(int l) const { return r->d[l]; }
};

template <int NT, int NTH, int MINB>
__global__ void __launch_bounds__(NTH, MINB) k_solve_wb(SolveArgs a) {
  __shared__ sb::WbTable wt;
  __shared__ float2 wds[NT];
  const int slot = (int)(blockIdx.x / a.bpp);
  const long long off = (long long)(blockIdx.x % a.bpp) * NTH + threadIdx.x;
  const int k = a.t.order ? a.t.order[slot] : slot;
  const bool inv = a.t.inv[k] != 0;
  const bool valid = off < a.plane;
  const long long idx = (long long)k * a.plane + (valid ? off : 0);
  if (!inv) {
    if (!valid) return;
    float2 c6[6];
#pragma unroll
    for (int t = 0; t < 6; ++t) c6[t] = a.g.cov[t][idx];
    sb::prior_only<0>(a.c, c6);
    bool nonfinite = false;
#pragma unroll
    for (int t = 0; t < 6; ++t) { a.g.cov[t][idx] = c6[t]; nonfinite |= !sb::fin2(c6[t]); }
    if (a.counters) sb::count(a.counters, false, nonfinite);
    return;
  }
  float2 c6[6], ec = make_float2(0.f, 0.f);
  RegIn<NT> in;
  if (valid) {
#pragma unroll
    for (int t = 0; t < 6; ++t) c6[t] = a.g.cov[t][idx];
    ec = a.g.err[idx];
#pragma unroll
    for (int q = 0; q < 3; ++q) in.m[q] = a.g.mu[q][idx];
#pragma unroll
    for (int l = 0; l < NT; ++l) in.d[l] = a.g.data[l][idx];
  }
  {
    // the rows i < NT of T (NT entries each), W and H, m, ok
    const sb::WbTable &src = a.wb[k];
    for (int e = threadIdx.x; e < NT * NT; e += NTH) wt.T[e / NT][e % NT] = src.T[e / NT][e % NT];
    for (int e = threadIdx.x; e < NT * 3; e += NTH) wt.W[e / 3][e % 3] = src.W[e / 3][e % 3];
    for (int e = threadIdx.x; e < NT * 9; e += NTH) wt.H[e / 9][e % 9] = src.H[e / 9][e % 9];
    if (threadIdx.x < NT) {
      wt.m[threadIdx.x] = src.m[threadIdx.x];
      wds[threadIdx.x] = a.t.wd[(long long)k * NT + threadIdx.x];
    }
    if (threadIdx.x == 0) wt.ok = src.ok;
  }
  __syncthreads();
  double L[6], cw[NT];
  bool ok = true;
  if (valid) {
    const sb::Sym3d S = sb::prior_exact(c6, a.c.var0);
    ok = wt.ok != 0;
    ok = sb::chol3(S, L) && ok;
    ok = sb::wb_weights<NT>(wt, fabs((double)ec.x), cw) && ok;
  }
  if (__syncthreads_or(!ok)) {
    if (threadIdx.x == 0) {
      const unsigned long long i = atomicAdd(&a.counters->deferred, 1ull);
      a.list[i] = (int)blockIdx.x;
    }
    return;
  }
  if (!valid) return;
  const bool fin = sb::solve_bin_wb<NT>(wt, a.c, wds, L, cw, a.g, idx, RegInAcc<NT>{&in});
  sb::count(a.counters, false, !fin);
}

// Per-plane Woodbury tables, one thread per kz plane.
template <int NT>
__global__ void k_kz_wb(SolveConsts c, KzTables t, int nzp) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nzp) return;
  sb::WbTable *w = reinterpret_cast<sb::WbTable *>(t.wb) + k;
  const long long o = (long long)k * NT;
  sb::WbTable tmp;
  sb::wb_table_fill<NT>(tmp, c, t.wd + o, t.e1 + o, t.e2 + o, t.e3 + o);
  if (!t.inv[k]) tmp.ok = 0;
  *w = tmp;
}

template <int NTH, int MINB>
int launch_solve_wb(SolveArgs a, int nt, cudaStream_t s) {
  a.bpp = (a.plane + NTH - 1) / NTH;
  const long long nblk = a.bpp * a.nslots;
  if (nblk > a.t.defer_n || nblk >= (1LL << 31) || !a.counters) return CRAVA_GPU_ERR_ARG;
  a.wb = reinterpret_cast<const sb::WbTable *>(a.t.wb);
  a.list = a.t.defer_list;
  dim3 grd((unsigned)nblk);
  // the deferred blocks: the square-root form, on a fixed grid of resident
  // blocks (k_solve_sq's shape 3: four 128-thread blocks per SM)
  int dev = 0, sms = 0;
  CRAVA_CUDA_TRY(cudaGetDevice(&dev));
  CRAVA_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const unsigned g2 = (unsigned)std::min<long long>(nblk, 4LL * sms);
  int rc;
#define CRAVA_WB_CASE(N)                                                                           \
  case N: {                                                                                        \
    k_solve_wb<N, NTH, MINB><<<grd, NTH, 0, s>>>(a);                                               \
    CRAVA_LAUNCH_CHECK();                                                                          \
    const size_t smem = SqSmem<N, 0, NTH, true>::bytes;                                            \
    if ((rc = func_smem((const void *)k_solve_sq_list<N, NTH, 4>, smem))) return rc;               \
    k_solve_sq_list<N, NTH, 4><<<g2, NTH, smem, s>>>(a);                                           \
    CRAVA_LAUNCH_CHECK();                                                                          \
    break;                                                                                         \
  }
  switch (nt) {
    CRAVA_WB_CASE(1) CRAVA_WB_CASE(2) CRAVA_WB_CASE(3) CRAVA_WB_CASE(4)
    CRAVA_WB_CASE(5) CRAVA_WB_CASE(6) CRAVA_WB_CASE(7) CRAVA_WB_CASE(8)
    default: return CRAVA_GPU_ERR_ARG;
  }
#undef CRAVA_WB_CASE
  return CRAVA_GPU_OK;
}

// Launch shape of the square-root solve: 0 the factor in shared memory
// (256 threads, two blocks per SM), 1 in registers with 128 threads and
// three blocks per SM (up to 170 registers), 2 in registers with 256
// threads and one block per SM (up to 255 registers), 3 in registers with
// 128 threads and four blocks per SM (up to 128 registers); 4 and 5 the
// pipelined kernel (k_solve_pf) with 128 threads, four blocks per SM and 4
// or 8 bins per thread.  Measured at 256x256x512x5 (B200, one stream),
// FP64 / mixed: 1.34 / 1.14 ms (shape 0), 1.34 / 1.23 (1), 1.76 / 1.74 (2),
// 1.17 / 1.06 (3), 1.03 / 1.11 (4), 1.01 / 1.09 (5).  The FP64 form is
// latency-bound on its global loads, which the pipelined kernel hides; the
// mixed form carries the FP32 factor and the FP64 refinement operands in
// registers, and the staging buffers cost it more occupancy than they
// save.  Shape 6 is the FP64 solve in the Woodbury form (k_solve_wb, 128
// threads, six blocks per SM), with the square-root form of shape 3 for the
// blocks it defers; it needs the context's Woodbury tables (not built for
// the allocation-free entry point).  Defaults: shape 6 for FP64 where the
// tables exist, else 5; shape 3 for mixed.  The context's tuning
// (SolveConsts::solve_shape) picks one explicitly, and CRAVA_SOLVE_SHAPE
// (0-6) overrides the built-in choice for measurements.
static int solve_shape_override() {
  static int v = -2;
  if (v == -2) {
    const char *e = getenv("CRAVA_SOLVE_SHAPE");
    v = e ? atoi(e) : -1;
    if (v < 0 || v > 8) v = -1;
  }
  return v;
}

template <int PREC>
int launch_solve_sq_shape(const SolveArgs &a, int nt, cudaStream_t s) {
  int shape = a.c.solve_shape >= 0 ? a.c.solve_shape : solve_shape_override();
  // the Woodbury form (FP64 only) needs the context's tables and flags
  const bool wb = PREC == 0 && a.t.wb && a.t.defer_list && a.counters;
  if (shape < 0) shape = PREC == 0 ? (wb ? 6 : 5) : 3;
  if (shape >= 6 && !wb) shape = PREC == 0 ? 5 : 3;
  switch (shape) {
    case 6: return launch_solve_wb<128, 6>(a, nt, s);
    case 7: return launch_solve_wb<128, 5>(a, nt, s);
    case 8: return launch_solve_wb<128, 4>(a, nt, s);
    case 0: return launch_solve_sq<PREC, 256, 2, false>(a, nt, s);
    case 1: return launch_solve_sq<PREC, 128, 3, true>(a, nt, s);
    case 2: return launch_solve_sq<PREC, 256, 1, true>(a, nt, s);
    case 4: return launch_solve_pf<PREC, 128, 4, 4>(a, nt, s);
    case 5: return launch_solve_pf<PREC, 128, 4, 8>(a, nt, s);
    default: return launch_solve_sq<PREC, 128, 4, true>(a, nt, s);
  }
}

}  // namespace

int kz_tables_alloc(int nzp, int nt, KzTables *t) {
  size_t n = (size_t)nzp * nt;
  CRAVA_CUDA_TRY(cudaMalloc(&t->wd, n * sizeof(float2)));
  CRAVA_CUDA_TRY(cudaMalloc(&t->e1, n * sizeof(float2)));
  CRAVA_CUDA_TRY(cudaMalloc(&t->e2, n * sizeof(float2)));
  CRAVA_CUDA_TRY(cudaMalloc(&t->e3, n * sizeof(float)));
  CRAVA_CUDA_TRY(cudaMalloc(&t->inv, (size_t)nzp * sizeof(int)));
  return CRAVA_GPU_OK;
}

void kz_tables_free(KzTables *t) {
  cudaFree(t->wd); cudaFree(t->e1); cudaFree(t->e2); cudaFree(t->e3); cudaFree(t->inv);
  cudaFree(t->order);
  cudaFree(t->order_inv);
  cudaFree(t->wb);
  cudaFree(t->defer_list);
  *t = KzTables{};
}

int kz_woodbury_alloc(int nzp, long long plane, KzTables *t) {
  const long long nblk = (plane + 127) / 128 * nzp;
  CRAVA_CUDA_TRY(cudaMalloc(&t->wb, (size_t)nzp * sizeof(sb::WbTable)));
  CRAVA_CUDA_TRY(cudaMalloc(&t->defer_list, (size_t)nblk * sizeof(int)));
  t->defer_n = nblk;
  return CRAVA_GPU_OK;
}

int kz_woodbury_build(const SolveConsts &c, int nzp, const KzTables &t, cudaStream_t s) {
  if (!t.wb) return CRAVA_GPU_OK;
  const int nth = 64, nb = (nzp + nth - 1) / nth;
  switch (c.nt) {
#define CRAVA_KWB(N) case N: k_kz_wb<N><<<nb, nth, 0, s>>>(c, t, nzp); break;
    CRAVA_KWB(1) CRAVA_KWB(2) CRAVA_KWB(3) CRAVA_KWB(4) CRAVA_KWB(5) CRAVA_KWB(6) CRAVA_KWB(7) CRAVA_KWB(8)
#undef CRAVA_KWB
    default: return CRAVA_GPU_ERR_ARG;
  }
  CRAVA_LAUNCH_CHECK();
  return CRAVA_GPU_OK;
}

int kz_order_build(int nzp, KzTables *t, cudaStream_t s, int *n_inverted) {
  std::vector<int> inv(nzp), order;
  CRAVA_CUDA_TRY(cudaMemcpyAsync(inv.data(), t->inv, sizeof(int) * nzp, cudaMemcpyDeviceToHost, s));
  CRAVA_CUDA_TRY(cudaStreamSynchronize(s));
  std::vector<int> heavy, light;
  for (int k = 0; k < nzp; ++k) (inv[k] ? heavy : light).push_back(k);
  const long long nh = (long long)heavy.size();
  if (n_inverted) *n_inverted = (int)nh;
  size_t ih = 0, il = 0;
  for (long long i = 0; i < nzp; ++i) {
    // Bresenham: the i-th slot takes a heavy plane when the heavy share so
    // far falls behind nh / nzp
    const bool take_heavy = ih < heavy.size() && ((long long)ih * nzp < (i + 1) * nh || il == light.size());
    order.push_back(take_heavy ? heavy[ih++] : light[il++]);
  }
  if (!t->order) CRAVA_CUDA_TRY(cudaMalloc(&t->order, sizeof(int) * nzp));
  if (!t->order_inv) CRAVA_CUDA_TRY(cudaMalloc(&t->order_inv, sizeof(int) * nzp));
  CRAVA_CUDA_TRY(cudaMemcpyAsync(t->order, order.data(), sizeof(int) * nzp, cudaMemcpyHostToDevice, s));
  if (nh) CRAVA_CUDA_TRY(cudaMemcpyAsync(t->order_inv, heavy.data(), sizeof(int) * nh, cudaMemcpyHostToDevice, s));
  CRAVA_CUDA_TRY(cudaStreamSynchronize(s));
  t->n_inv = (int)nh;
  return CRAVA_GPU_OK;
}

int kz_tables_build(const crava_gpu_params &p, KzTables *t, cudaStream_t s) {
  const int nzp = p.nzp, nt = p.ntheta;
  float *dw = nullptr, *dn = nullptr;
  CRAVA_CUDA_TRY(cudaMalloc(&dw, sizeof(float) * nzp * nt));
  CRAVA_CUDA_TRY(cudaMemcpyAsync(dw, p.wavelet, sizeof(float) * nzp * nt, cudaMemcpyHostToDevice, s));
  if (p.wavelet_norm) {
    CRAVA_CUDA_TRY(cudaMalloc(&dn, sizeof(float) * nt));
    CRAVA_CUDA_TRY(cudaMemcpyAsync(dn, p.wavelet_norm, sizeof(float) * nt, cudaMemcpyHostToDevice, s));
  }
  const int nth = 256;
  const int cnzp = nzp / 2 + 1;
  size_t smem = sizeof(double) * (2 * nzp + 2 * nth) + sizeof(float2) * 2 * cnzp + sizeof(float) * 4 * nzp;
  if (smem > 48 * 1024)
    CRAVA_CUDA_TRY(cudaFuncSetAttribute(k_kz_tables, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_kz_tables<<<nt, nth, smem, s>>>(dw, dn, p.wavelet_norm != nullptr, nzp, nt, p.nz, p.lz,
                                    p.min_rel_thick, p.low_cut, p.high_cut, p.thickness_mode, *t);
  cudaError_t le = cudaGetLastError();
  cudaError_t se = cudaStreamSynchronize(s);
  cudaFree(dw);
  if (dn) cudaFree(dn);
  if (le != cudaSuccess) { set_last_error(le, "k_kz_tables", __FILE__, __LINE__); return CRAVA_GPU_ERR_CUDA; }
  if (se != cudaSuccess) { set_last_error(se, "k_kz_tables sync", __FILE__, __LINE__); return CRAVA_GPU_ERR_CUDA; }
  note_launch();
  return CRAVA_GPU_OK;
}

int kz_tables_build_device(const crava_gpu_params &p, const float *d_wavelet,
                           const float *d_norm, KzTables *t, cudaStream_t s) {
  const int nzp = p.nzp, nt = p.ntheta;
  const int nth = 256;
  const int cnzp = nzp / 2 + 1;
  size_t smem = sizeof(double) * (2 * nzp + 2 * nth) + sizeof(float2) * 2 * cnzp + sizeof(float) * 4 * nzp;
  if (smem > 48 * 1024)
    CRAVA_CUDA_TRY(cudaFuncSetAttribute(k_kz_tables, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_kz_tables<<<nt, nth, smem, s>>>(d_wavelet, d_norm, d_norm != nullptr, nzp, nt, p.nz, p.lz,
                                    p.min_rel_thick, p.low_cut, p.high_cut, p.thickness_mode, *t);
  CRAVA_LAUNCH_CHECK();
  return CRAVA_GPU_OK;
}

int posterior_solve(const SolveConsts &c, const KzTables &t, const SolveGrids &g,
                    long long csize, long long plane, int precision,
                    DevCounters *counters, cudaStream_t s, bool gated_done) {
  if (precision == CRAVA_SOLVE_FP32) {
    if (gated_done) return CRAVA_GPU_ERR_ARG;  // the reference-order kernel visits every bin
    return posterior_solve_fp32ref(c, t, g, csize, plane, counters, s);
  }
  SolveArgs a;
  a.c = c; a.g = g; a.t = t; a.csize = csize; a.plane = plane; a.counters = counters;
  a.bpp = (plane + kThreads - 1) / kThreads;
  a.nslots = csize / plane;
  if (gated_done) {
    if (t.n_inv < 0 || !t.order_inv) return CRAVA_GPU_ERR_ARG;
    a.t.order = t.order_inv;
    a.nslots = t.n_inv;
    if (a.nslots == 0) return CRAVA_GPU_OK;  // no inverted plane: nothing left to solve
  }
  // the square-root form (one kz plane per CTA)
  if (precision == CRAVA_SOLVE_FP64) return launch_solve_sq_shape<0>(a, c.nt, s);
  if (precision == CRAVA_SOLVE_MIXED) return launch_solve_sq_shape<1>(a, c.nt, s);
  return CRAVA_GPU_ERR_ARG;
}

}  // namespace crava

namespace crava {

namespace {

__global__ void __launch_bounds__(1024) k_gated_nonfinite(unsigned *bits, long long nwords, unsigned *any,
                                                          DevCounters *ctr) {
  if (*(volatile unsigned *)any == 0u) return;  // every thread reads the flag before thread 0 clears it
  unsigned long long n = 0;
  for (long long i = threadIdx.x; i < nwords; i += blockDim.x) {
    const unsigned w = bits[i];
    if (w) {
      n += (unsigned long long)__popc(w);
      bits[i] = 0u;
    }
  }
  if (n) atomicAdd(&ctr->nonfinite, n);
  __syncthreads();
  if (threadIdx.x == 0) *any = 0u;
}

}  // namespace

int gated_nonfinite_count(unsigned *nf_bits, long long nwords, unsigned *nf_any, DevCounters *counters,
                          cudaStream_t s) {
  k_gated_nonfinite<<<1, 1024, 0, s>>>(nf_bits, nwords, nf_any, counters);
  CRAVA_LAUNCH_CHECK();
  return CRAVA_GPU_OK;
}

}  // namespace crava
