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

#include "solve.cuh"

namespace crava {

namespace {

constexpr int kThreads = 256;
constexpr double kTol = 1e-20;  // libs/lib/lib_matr.c:20

__host__ __device__ constexpr int tri(int i, int j) { return i * (i + 1) / 2 + j; }

// ------------------------------------------------------------------ tables
__global__ void k_kz_tables(const float *__restrict__ wav,
                            const float *__restrict__ wnorm_in, int has_norm,
                            int nzp, int nt, int nz, double lz, double mrt,
                            float low_cut, float high_cut, KzTables t) {
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
    float2 kw = make_float2(ca.x, -ca.y);  // fillkW (src/crava.cpp:1336-1344)
    float2 wd = make_float2(kD.x * kw.x - kD.y * kw.y, kD.x * kw.y + kD.y * kw.x);
    const long long o = (long long)k * nt + l;
    t.wd[o] = wd;
    t.e1[o] = make_float2(ca.x / wn, -(ca.y / wn));  // fillkWNorm (:1346-1355)
    t.e2[o] = make_float2(cg.x / gn, -(cg.y / gn));
    t.e3[o] = 1.0f;
    if (l == 0) {
      int mk = k < nzp - k ? k : nzp - k;
      float rf = (float)((nz * 1000.0f) / (lz * nzp) * mk);  // src/crava.cpp:1044
      t.inv[k] = (rf > low_cut * mrt) && (rf < high_cut);
    }
  }
}

// ------------------------------------------------------------------ helpers
struct Sym3d { double s00, s11, s22, s01, s02, s12; };

__device__ __forceinline__ double sget(const Sym3d &s, int a, int b) {
  if (a > b) { int t = a; a = b; b = t; }
  return a == 0 ? (b == 0 ? s.s00 : b == 1 ? s.s01 : s.s02) : a == 1 ? (b == 1 ? s.s11 : s.s12) : s.s22;
}

// getNextParameterCovariance in double: S_pq = |Re(c)/v| v (no division if v == 0).
__device__ __forceinline__ Sym3d prior_d(const float2 c6[6], const double v[6]) {
  double r[6];
#pragma unroll
  for (int t = 0; t < 6; ++t) {
    double x = c6[t].x;
    r[t] = v[t] != 0.0 ? fabs(x / v[t]) * v[t] : fabs(x);
  }
  return Sym3d{r[0], r[1], r[2], r[3], r[4], r[5]};
}

// Same in float, with the reference's operations (float divide, |.|, float multiply).
__device__ __forceinline__ void prior_f(const float2 c6[6], const double v[6], float r[6]) {
#pragma unroll
  for (int t = 0; t < 6; ++t) {
    float vf = (float)v[t];
    float x = c6[t].x;
    if (v[t] != 0.0) x = x / vf;
    r[t] = fabsf(x) * vf;
  }
}

// Hermitian Cholesky M = L L^H on the lower triangle (tri() indexing), with
// the reference's failure rules applied to M / M00.
template <int NT, typename T2, typename T>
__device__ __forceinline__ bool cholesky(T2 *L) {
  const T factor = L[0].x;
  if (!(factor > T(0))) return false;
  const T tol = (T)kTol * factor;
#pragma unroll
  for (int i = 0; i < NT; ++i) {
    if (!(L[tri(i, i)].x > tol)) return false;
#pragma unroll
    for (int j = 0; j < i; ++j) {
      T2 s = L[tri(i, j)];
#pragma unroll
      for (int k = 0; k < j; ++k) {
        T2 a = L[tri(i, k)], b = L[tri(j, k)];
        s.x -= a.x * b.x + a.y * b.y;
        s.y -= a.y * b.x - a.x * b.y;
      }
      T inv = T(1) / L[tri(j, j)].x;
      s.x *= inv; s.y *= inv;
      L[tri(i, j)] = s;
    }
    T d = L[tri(i, i)].x;
#pragma unroll
    for (int k = 0; k < i; ++k) d -= L[tri(i, k)].x * L[tri(i, k)].x + L[tri(i, k)].y * L[tri(i, k)].y;
    if (!(d > tol)) return false;
    L[tri(i, i)].x = sqrt(d);
    L[tri(i, i)].y = T(0);
  }
  return true;
}

// Solves L L^H X = B in place for the 3 columns of B.
template <int NT, typename T2, typename T>
__device__ __forceinline__ void chol_solve3(const T2 *L, T2 (*B)[3]) {
#pragma unroll
  for (int c = 0; c < 3; ++c) {
#pragma unroll
    for (int i = 0; i < NT; ++i) {
      T2 s = B[i][c];
#pragma unroll
      for (int j = 0; j < i; ++j) {
        T2 l = L[tri(i, j)], x = B[j][c];
        s.x -= l.x * x.x - l.y * x.y;
        s.y -= l.x * x.y + l.y * x.x;
      }
      T inv = T(1) / L[tri(i, i)].x;
      B[i][c].x = s.x * inv; B[i][c].y = s.y * inv;
    }
#pragma unroll
    for (int i = NT - 1; i >= 0; --i) {
      T2 s = B[i][c];
#pragma unroll
      for (int j = i + 1; j < NT; ++j) {
        T2 l = L[tri(j, i)], x = B[j][c];  // conj(l) * x
        s.x -= l.x * x.x + l.y * x.y;
        s.y -= l.x * x.y - l.y * x.x;
      }
      T inv = T(1) / L[tri(i, i)].x;
      B[i][c].x = s.x * inv; B[i][c].y = s.y * inv;
    }
  }
}

struct SolveArgs {
  SolveConsts c;
  SolveGrids g;
  KzTables t;
  long long csize, plane;
  DevCounters *counters;
};

__device__ __forceinline__ void count(DevCounters *ctr, bool fail, bool nonfinite) {
  unsigned m = __activemask();
  unsigned bf = __ballot_sync(m, fail), bn = __ballot_sync(m, nonfinite);
  int leader = __ffs(m) - 1;
  if ((threadIdx.x & 31) == leader) {
    if (bf) atomicAdd(&ctr->chol_fail, (unsigned long long)__popc(bf));
    if (bn) atomicAdd(&ctr->nonfinite, (unsigned long long)__popc(bn));
  }
}

__device__ __forceinline__ bool fin2(float2 v) { return isfinite(v.x) && isfinite(v.y); }

// PREC 0: FP64 throughout.  PREC 1: FP32 build and factorisation, one FP64
// refinement step on the residual K S - M X0, FP64 Schur update and mean.
template <int NT, int PREC>
__global__ void __launch_bounds__(kThreads) k_solve(SolveArgs a) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= a.csize) return;
  const int k = (int)(idx / a.plane);
  const SolveConsts &c = a.c;

  float2 mu[3], d[NT], c6[6];
#pragma unroll
  for (int q = 0; q < 3; ++q) mu[q] = a.g.mu[q][idx];
#pragma unroll
  for (int l = 0; l < NT; ++l) d[l] = a.g.data[l][idx];
#pragma unroll
  for (int t = 0; t < 6; ++t) c6[t] = a.g.cov[t][idx];
  const float2 ec = a.g.err[idx];
  const bool inv = a.t.inv[k] != 0;

  const Sym3d S = prior_d(c6, c.var0);
  float2 out_mu[3], out_r[NT];
  double2 Sp[6];  // posterior (0,0) (1,1) (2,2) (0,1) (0,2) (1,2)
  const int pa[6] = {0, 1, 2, 0, 0, 1}, pb[6] = {0, 1, 2, 1, 2, 2};
  bool fail = false;
  bool solved = false;
  if (PREC == 1) {
    float sf[6];
    prior_f(c6, c.var0, sf);
#pragma unroll
    for (int t = 0; t < 6; ++t) Sp[t] = make_double2(sf[t], 0.0);
  } else {
#pragma unroll
    for (int t = 0; t < 6; ++t) Sp[t] = make_double2(sget(S, pa[t], pb[t]), 0.0);
  }

  if (inv) {
    const float2 *wdk = a.t.wd + (long long)k * NT;
    const float2 *e1k = a.t.e1 + (long long)k * NT;
    const float2 *e2k = a.t.e2 + (long long)k * NT;
    const float *e3k = a.t.e3 + (long long)k * NT;
    float2 wd[NT], e1[NT], e2[NT];
    float e3[NT];
#pragma unroll
    for (int l = 0; l < NT; ++l) { wd[l] = __ldg(wdk + l); e1[l] = __ldg(e1k + l); e2[l] = __ldg(e2k + l); e3[l] = __ldg(e3k + l); }
    const double lam = fabs((double)ec.x);
    const double cc = 0.5 * (1.0 - (double)c.wnc);

    // A S (real, double) and K S = diag(wd) A S
    double AS[NT][3];
#pragma unroll
    for (int l = 0; l < NT; ++l)
#pragma unroll
      for (int q = 0; q < 3; ++q)
        AS[l][q] = (double)c.A[l][0] * sget(S, 0, q) + (double)c.A[l][1] * sget(S, 1, q) + (double)c.A[l][2] * sget(S, 2, q);
    double2 X[NT][3];

    if (PREC == 0) {
      double2 L[NT * (NT + 1) / 2];
#pragma unroll
      for (int l = 0; l < NT; ++l)
#pragma unroll
        for (int m = 0; m <= l; ++m) {
          double B = AS[l][0] * c.A[m][0] + AS[l][1] * c.A[m][1] + AS[l][2] * c.A[m][2];
          double2 w = dmulc(make_double2(wd[l].x, wd[l].y), make_double2(wd[m].x, wd[m].y));
          double th = c.theta[l][m];
          double2 n1 = dmulc(make_double2(e1[l].x, e1[l].y), make_double2(e1[m].x, e1[m].y));
          double2 n2 = dmulc(make_double2(e2[l].x, e2[l].y), make_double2(e2[m].x, e2[m].y));
          double f = cc * th * lam;
          double2 v = make_double2(w.x * B + f * (n1.x + n2.x), w.y * B + f * (n1.y + n2.y));
          if (l == m) { v.x += (double)c.wnc * th * (double)e3[l] * (double)e3[l]; v.y = 0.0; }
          L[tri(l, m)] = v;
        }
#pragma unroll
      for (int l = 0; l < NT; ++l)
#pragma unroll
        for (int q = 0; q < 3; ++q) X[l][q] = make_double2(wd[l].x * AS[l][q], wd[l].y * AS[l][q]);
      if (cholesky<NT, double2, double>(L)) {
        chol_solve3<NT, double2, double>(L, X);
        solved = true;
      } else {
        fail = true;
      }
    } else {
      // FP32 build and factorisation
      float sf[6];
      prior_f(c6, c.var0, sf);
      auto sgf = [&](int p, int q) -> float {
        if (p > q) { int t = p; p = q; q = t; }
        return p == 0 ? (q == 0 ? sf[0] : q == 1 ? sf[3] : sf[4]) : p == 1 ? (q == 1 ? sf[1] : sf[5]) : sf[2];
      };
      float ASf[NT][3];
#pragma unroll
      for (int l = 0; l < NT; ++l)
#pragma unroll
        for (int q = 0; q < 3; ++q)
          ASf[l][q] = c.A[l][0] * sgf(0, q) + c.A[l][1] * sgf(1, q) + c.A[l][2] * sgf(2, q);
      float2 Lf[NT * (NT + 1) / 2];
      const float ff = (float)(cc * lam);
#pragma unroll
      for (int l = 0; l < NT; ++l)
#pragma unroll
        for (int m = 0; m <= l; ++m) {
          float B = ASf[l][0] * c.A[m][0] + ASf[l][1] * c.A[m][1] + ASf[l][2] * c.A[m][2];
          float2 w = cmulc(wd[l], wd[m]);
          float th = (float)c.theta[l][m];
          float2 n1 = cmulc(e1[l], e1[m]), n2 = cmulc(e2[l], e2[m]);
          float f = ff * th;
          float2 v = make_float2(w.x * B + f * (n1.x + n2.x), w.y * B + f * (n1.y + n2.y));
          if (l == m) { v.x += c.wnc * th * e3[l] * e3[l]; v.y = 0.f; }
          Lf[tri(l, m)] = v;
        }
      float2 Xf[NT][3];
#pragma unroll
      for (int l = 0; l < NT; ++l)
#pragma unroll
        for (int q = 0; q < 3; ++q) Xf[l][q] = make_float2(wd[l].x * ASf[l][q], wd[l].y * ASf[l][q]);
      if (cholesky<NT, float2, float>(Lf)) {
        chol_solve3<NT, float2, float>(Lf, Xf);
        // FP64 residual of the exact system: Rd = KS - M X0.
        float2 Rf[NT][3];
#pragma unroll
        for (int l = 0; l < NT; ++l) {
          double2 acc[3];
#pragma unroll
          for (int q = 0; q < 3; ++q) acc[q] = make_double2(wd[l].x * AS[l][q], wd[l].y * AS[l][q]);
#pragma unroll
          for (int m = 0; m < NT; ++m) {
            // M_lm in double (Hermitian: M_lm = conj(M_ml))
            double B = AS[l][0] * c.A[m][0] + AS[l][1] * c.A[m][1] + AS[l][2] * c.A[m][2];
            double2 w = dmulc(make_double2(wd[l].x, wd[l].y), make_double2(wd[m].x, wd[m].y));
            double th = c.theta[l][m];
            double2 n1 = dmulc(make_double2(e1[l].x, e1[l].y), make_double2(e1[m].x, e1[m].y));
            double2 n2 = dmulc(make_double2(e2[l].x, e2[l].y), make_double2(e2[m].x, e2[m].y));
            double f = cc * th * lam;
            double2 Mv = make_double2(w.x * B + f * (n1.x + n2.x), w.y * B + f * (n1.y + n2.y));
            if (l == m) { Mv.x += (double)c.wnc * th * (double)e3[l] * (double)e3[l]; Mv.y = 0.0; }
#pragma unroll
            for (int q = 0; q < 3; ++q) {
              double2 x = make_double2(Xf[m][q].x, Xf[m][q].y);
              acc[q] = dsub(acc[q], dmul(Mv, x));
            }
          }
#pragma unroll
          for (int q = 0; q < 3; ++q) Rf[l][q] = make_float2((float)acc[q].x, (float)acc[q].y);
        }
        chol_solve3<NT, float2, float>(Lf, Rf);
#pragma unroll
        for (int l = 0; l < NT; ++l)
#pragma unroll
          for (int q = 0; q < 3; ++q)
            X[l][q] = make_double2((double)Xf[l][q].x + (double)Rf[l][q].x, (double)Xf[l][q].y + (double)Rf[l][q].y);
        solved = true;
#pragma unroll
        for (int t = 0; t < 6; ++t) Sp[t] = make_double2(sget(S, pa[t], pb[t]), 0.0);
      } else {
        fail = true;
      }
    }

    if (solved) {
      // S_post = S - (KS)^H X   (FP64)
#pragma unroll
      for (int t = 0; t < 6; ++t) {
        const int p = pa[t], q = pb[t];
        double2 r = make_double2(0.0, 0.0);
#pragma unroll
        for (int l = 0; l < NT; ++l) {
          double2 ks = make_double2(wd[l].x * AS[l][p], wd[l].y * AS[l][p]);
          r = dadd(r, dmulc(X[l][q], ks));  // conj(ks) * X
        }
        Sp[t] = make_double2(Sp[t].x - r.x, Sp[t].y - r.y);
      }
      // mean and residual
      double2 v[NT];
#pragma unroll
      for (int l = 0; l < NT; ++l) {
        double2 km = make_double2(0, 0);
#pragma unroll
        for (int q = 0; q < 3; ++q) km = dadd(km, make_double2(c.A[l][q] * (double)mu[q].x, c.A[l][q] * (double)mu[q].y));
        km = dmul(make_double2(wd[l].x, wd[l].y), km);
        v[l] = make_double2((double)d[l].x - km.x, (double)d[l].y - km.y);
      }
      double2 mp[3];
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        double2 s = make_double2(mu[q].x, mu[q].y);
#pragma unroll
        for (int l = 0; l < NT; ++l) s = dadd(s, dmulc(v[l], X[l][q]));  // conj(X) v
        mp[q] = s;
        out_mu[q] = make_float2((float)s.x, (float)s.y);
      }
#pragma unroll
      for (int l = 0; l < NT; ++l) {
        double2 km = make_double2(0, 0);
#pragma unroll
        for (int q = 0; q < 3; ++q) km = dadd(km, make_double2(c.A[l][q] * mp[q].x, c.A[l][q] * mp[q].y));
        km = dmul(make_double2(wd[l].x, wd[l].y), km);
        out_r[l] = make_float2((float)((double)d[l].x - km.x), (float)((double)d[l].y - km.y));
      }
    }
  }
  if (!solved) {
#pragma unroll
    for (int q = 0; q < 3; ++q) out_mu[q] = mu[q];
#pragma unroll
    for (int l = 0; l < NT; ++l) out_r[l] = d[l];
  }
  bool nonfinite = false;
#pragma unroll
  for (int q = 0; q < 3; ++q) { a.g.mu[q][idx] = out_mu[q]; nonfinite |= !fin2(out_mu[q]); }
#pragma unroll
  for (int l = 0; l < NT; ++l) { a.g.data[l][idx] = out_r[l]; nonfinite |= !fin2(out_r[l]); }
#pragma unroll
  for (int t = 0; t < 6; ++t) {
    float2 o = make_float2((float)Sp[t].x, (float)Sp[t].y);
    a.g.cov[t][idx] = o;
    nonfinite |= !fin2(o);
  }
  if (a.counters) count(a.counters, fail, nonfinite);
}

template <int PREC>
int launch_solve(const SolveArgs &a, int nt, cudaStream_t s) {
  dim3 grd((unsigned)((a.csize + kThreads - 1) / kThreads));
  switch (nt) {
    case 1: k_solve<1, PREC><<<grd, kThreads, 0, s>>>(a); break;
    case 2: k_solve<2, PREC><<<grd, kThreads, 0, s>>>(a); break;
    case 3: k_solve<3, PREC><<<grd, kThreads, 0, s>>>(a); break;
    case 4: k_solve<4, PREC><<<grd, kThreads, 0, s>>>(a); break;
    case 5: k_solve<5, PREC><<<grd, kThreads, 0, s>>>(a); break;
    case 6: k_solve<6, PREC><<<grd, kThreads, 0, s>>>(a); break;
    case 7: k_solve<7, PREC><<<grd, kThreads, 0, s>>>(a); break;
    case 8: k_solve<8, PREC><<<grd, kThreads, 0, s>>>(a); break;
    default: return CRAVA_GPU_ERR_ARG;
  }
  CRAVA_LAUNCH_CHECK();
  return CRAVA_GPU_OK;
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
  *t = KzTables{};
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
                                    p.min_rel_thick, p.low_cut, p.high_cut, *t);
  cudaError_t le = cudaGetLastError();
  cudaError_t se = cudaStreamSynchronize(s);
  cudaFree(dw);
  if (dn) cudaFree(dn);
  if (le != cudaSuccess) { set_last_error(le, "k_kz_tables", __FILE__, __LINE__); return CRAVA_GPU_ERR_CUDA; }
  if (se != cudaSuccess) { set_last_error(se, "k_kz_tables sync", __FILE__, __LINE__); return CRAVA_GPU_ERR_CUDA; }
  note_launch();
  return CRAVA_GPU_OK;
}

int posterior_solve(const SolveConsts &c, const KzTables &t, const SolveGrids &g,
                    long long csize, long long plane, int precision,
                    DevCounters *counters, cudaStream_t s) {
  if (precision == CRAVA_SOLVE_FP32) return posterior_solve_fp32ref(c, t, g, csize, plane, counters, s);
  SolveArgs a;
  a.c = c; a.g = g; a.t = t; a.csize = csize; a.plane = plane; a.counters = counters;
  if (precision == CRAVA_SOLVE_FP64) return launch_solve<0>(a, c.nt, s);
  if (precision == CRAVA_SOLVE_MIXED) return launch_solve<1>(a, c.nt, s);
  return CRAVA_GPU_ERR_ARG;
}

}  // namespace crava
