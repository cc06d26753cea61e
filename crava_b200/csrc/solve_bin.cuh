// solve_bin.cuh -- the per-bin posterior solve as a device function, shared
// by the standalone solve kernel (solve.cu) and the fused z-transform + solve
// kernel (unit.cu).  See solve.cu for the algebra and the reference lines.
#pragma once

#include <math.h>

#include "solve.cuh"

namespace crava {
namespace sb {

constexpr double kTol = 1e-20;  // libs/lib/lib_matr.c:20

__host__ __device__ constexpr int tri(int i, int j) { return i * (i + 1) / 2 + j; }

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
// the reference's failure rules applied to M / M00 (libs/lib/lib_matr.c:
// 103-105, 114, 145): M00 <= 0, or a diagonal entry or pivot of M / M00 <=
// 1e-20, fails.  The comparisons are the reference's (<=), so a NaN in M
// does not fail: it flows into the outputs as it does there.  The
// reciprocals of the diagonal of L are returned in rd (one division per
// column, reused by the substitutions).
template <int NT, typename T2, typename T, typename LA>
__device__ __forceinline__ bool cholesky(LA L, T *rd) {
  const T factor = L[0].x;
  if (factor <= T(0)) return false;
  const T tol = (T)kTol * factor;
#pragma unroll
  for (int i = 0; i < NT; ++i) {
    if (L[tri(i, i)].x <= tol) return false;
#pragma unroll
    for (int j = 0; j < i; ++j) {
      T2 s = L[tri(i, j)];
#pragma unroll
      for (int k = 0; k < j; ++k) {
        T2 a = L[tri(i, k)], b = L[tri(j, k)];
        s.x -= a.x * b.x + a.y * b.y;
        s.y -= a.y * b.x - a.x * b.y;
      }
      s.x *= rd[j]; s.y *= rd[j];
      L[tri(i, j)] = s;
    }
    T d = L[tri(i, i)].x;
#pragma unroll
    for (int k = 0; k < i; ++k) d -= L[tri(i, k)].x * L[tri(i, k)].x + L[tri(i, k)].y * L[tri(i, k)].y;
    if (d <= tol) return false;
    // one reciprocal square root gives both the pivot and its reciprocal
    const T r = rsqrt(d);
    L[tri(i, i)].x = d * r;
    L[tri(i, i)].y = T(0);
    rd[i] = r;
  }
  return true;
}

template <int NT, typename T2, typename T>
__device__ __forceinline__ bool cholesky(T2 *L) {
  T rd[NT];
  return cholesky<NT, T2, T, T2 *>(L, rd);
}

// A per-thread triangle held in shared memory, entries STRIDE apart
// (structure of arrays over the block: conflict-free, and it frees the
// registers of the factor).
template <typename T2, int STRIDE>
struct SmemTri {
  T2 *p;
  __device__ __forceinline__ T2 &operator[](int t) const { return p[t * STRIDE]; }
};

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

// FP64 form, one right-hand side at a time to bound register use: M (lower
// triangle, double) is built and factorised; then for each column q of
// K S the system M x = (K S)_q is solved, the posterior covariance entries
// (p, q), p <= q, are updated (S_pq - (KS)_p^H x) and the mean correction
// conj(x)^T (d - K mu) is accumulated.  Same algebra as the dense form.
template <int NT, typename LA, typename AA>
__device__ __forceinline__ bool solve_bin_fp64_in(LA L, AA AS, const SolveConsts &c,
                                                  const float2 *__restrict__ wdk,
                                                  const float2 *__restrict__ e1k,
                                                  const float2 *__restrict__ e2k,
                                                  const float *__restrict__ e3k, bool inv,
                                                  float2 mu[3], float2 d[NT], float2 c6[6], float2 ec) {
  const Sym3d S = prior_d(c6, c.var0);
  const int pa[6] = {0, 1, 2, 0, 0, 1}, pb[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
  for (int t = 0; t < 6; ++t) c6[t] = make_float2((float)sget(S, pa[t], pb[t]), 0.f);
  if (!inv) return false;
  // AS = A S (row l at AS[3 l .. 3 l + 2]), formed once
#pragma unroll
  for (int l = 0; l < NT; ++l)
#pragma unroll
    for (int p = 0; p < 3; ++p)
      AS[3 * l + p] = (double)c.A[l][0] * sget(S, 0, p) + (double)c.A[l][1] * sget(S, 1, p) +
                      (double)c.A[l][2] * sget(S, 2, p);
  {
    const double lam = fabs((double)ec.x);
    const double cc = 0.5 * (1.0 - (double)c.wnc) * lam;
#pragma unroll
    for (int l = 0; l < NT; ++l) {
      const double as0 = AS[3 * l], as1 = AS[3 * l + 1], as2 = AS[3 * l + 2];
      const float2 wl = __ldg(wdk + l), e1l = __ldg(e1k + l), e2l = __ldg(e2k + l);
#pragma unroll
      for (int m = 0; m <= l; ++m) {
        const double B = as0 * c.A[m][0] + as1 * c.A[m][1] + as2 * c.A[m][2];
        const float2 wm = __ldg(wdk + m), e1m = __ldg(e1k + m), e2m = __ldg(e2k + m);
        const double2 w = dmulc(make_double2(wl.x, wl.y), make_double2(wm.x, wm.y));
        const double2 n1 = dmulc(make_double2(e1l.x, e1l.y), make_double2(e1m.x, e1m.y));
        const double2 n2 = dmulc(make_double2(e2l.x, e2l.y), make_double2(e2m.x, e2m.y));
        const double f = cc * c.theta[l][m];
        double2 v = make_double2(w.x * B + f * (n1.x + n2.x), w.y * B + f * (n1.y + n2.y));
        if (l == m) {
          const double e3 = (double)__ldg(e3k + l);
          v.x += (double)c.wnc * c.theta[l][l] * e3 * e3;
          v.y = 0.0;
        }
        L[tri(l, m)] = v;
      }
    }
  }
  double rd[NT];
  if (!cholesky<NT, double2, double, LA>(L, rd)) return true;
  // residual of the prior mean, v = d - K mu, formed once
  double2 v[NT];
#pragma unroll
  for (int l = 0; l < NT; ++l) {
    double2 km = make_double2(0.0, 0.0);
#pragma unroll
    for (int r = 0; r < 3; ++r)
      km = dadd(km, make_double2(c.A[l][r] * (double)mu[r].x, c.A[l][r] * (double)mu[r].y));
    const float2 wl = __ldg(wdk + l);
    km = dmul(make_double2(wl.x, wl.y), km);
    v[l] = make_double2((double)d[l].x - km.x, (double)d[l].y - km.y);
  }
  double2 dm[3];  // mean corrections X^H v
  // one right-hand side at a time, loop kept rolled: the register budget
  // then allows two blocks per SM
#pragma unroll 1
  for (int q = 0; q < 3; ++q) {
    double2 x[NT];
#pragma unroll
    for (int l = 0; l < NT; ++l) {
      const double as = AS[3 * l + q];
      const float2 wl = __ldg(wdk + l);
      x[l] = make_double2(wl.x * as, wl.y * as);
    }
    // L y = x, then L^H x = y
#pragma unroll
    for (int i = 0; i < NT; ++i) {
      double2 s = x[i];
#pragma unroll
      for (int j = 0; j < i; ++j) {
        const double2 lij = L[tri(i, j)], xj = x[j];
        s.x -= lij.x * xj.x - lij.y * xj.y;
        s.y -= lij.x * xj.y + lij.y * xj.x;
      }
      x[i] = make_double2(s.x * rd[i], s.y * rd[i]);
    }
#pragma unroll
    for (int i = NT - 1; i >= 0; --i) {
      double2 s = x[i];
#pragma unroll
      for (int j = i + 1; j < NT; ++j) {
        const double2 lji = L[tri(j, i)], xj = x[j];  // conj(lji) * xj
        s.x -= lji.x * xj.x + lji.y * xj.y;
        s.y -= lji.x * xj.y - lji.y * xj.x;
      }
      x[i] = make_double2(s.x * rd[i], s.y * rd[i]);
    }
    // mean correction conj(x)^T v
    double2 acc = make_double2(0.0, 0.0);
#pragma unroll
    for (int l = 0; l < NT; ++l) acc = dadd(acc, dmulc(v[l], x[l]));
    if (q == 0) dm[0] = acc;
    else if (q == 1) dm[1] = acc;
    else dm[2] = acc;
    // posterior covariance entries (p, q), p <= q: S_pq - KS_p^H x with
    // KS = diag(w) AS, i.e. S_pq - sum_l AS_lp u_l, u = conj(w) x
#pragma unroll
    for (int l = 0; l < NT; ++l) {
      const float2 wl = __ldg(wdk + l);
      x[l] = make_double2(wl.x * x[l].x + wl.y * x[l].y, wl.x * x[l].y - wl.y * x[l].x);
    }
#pragma unroll
    for (int p = 0; p <= q; ++p) {
      double2 r = make_double2(0.0, 0.0);
#pragma unroll
      for (int l = 0; l < NT; ++l) {
        const double as = AS[3 * l + p];
        r.x += as * x[l].x;
        r.y += as * x[l].y;
      }
      const int t = p == q ? p : (p == 0 ? (q == 1 ? 3 : 4) : 5);
      c6[t] = make_float2((float)(sget(S, p, q) - r.x), (float)(-r.y));
    }
  }
  // residual d - K (mu + dm) = v - K dm; posterior mean mu + dm
#pragma unroll
  for (int l = 0; l < NT; ++l) {
    double2 km = make_double2(0.0, 0.0);
#pragma unroll
    for (int r = 0; r < 3; ++r) km = dadd(km, make_double2(c.A[l][r] * dm[r].x, c.A[l][r] * dm[r].y));
    const float2 wl = __ldg(wdk + l);
    km = dmul(make_double2(wl.x, wl.y), km);
    d[l] = make_float2((float)(v[l].x - km.x), (float)(v[l].y - km.y));
  }
#pragma unroll
  for (int q = 0; q < 3; ++q)
    mu[q] = make_float2((float)((double)mu[q].x + dm[q].x), (float)((double)mu[q].y + dm[q].y));
  return false;
}

template <int NT>
__device__ __forceinline__ bool solve_bin_fp64(const SolveConsts &c, const float2 *__restrict__ wdk,
                                               const float2 *__restrict__ e1k,
                                               const float2 *__restrict__ e2k,
                                               const float *__restrict__ e3k, bool inv,
                                               float2 mu[3], float2 d[NT], float2 c6[6], float2 ec) {
  double2 L[NT * (NT + 1) / 2];
  double AS[3 * NT];
  return solve_bin_fp64_in<NT, double2 *, double *>(L, AS, c, wdk, e1k, e2k, e3k, inv, mu, d, c6, ec);
}

// Mixed form, one right-hand side at a time: M is built in FP32 and
// factorised in FP32 (Lf); M is also kept in FP64 (Md, lower triangle) for
// the refinement residual.  For each column q of K S: x0 = M^-1 (KS)_q in
// FP32, r = (KS)_q - M x0 in FP64, x = x0 + M^-1 r (FP32 solve of r, FP64
// add); the posterior covariance entries S_pq - (KS)_p^H x and the mean
// correction are formed in FP64.
template <int NT, typename LAF, typename LAD, typename AA>
__device__ __forceinline__ bool solve_bin_mixed_in(LAF Lf, LAD Md, AA AS, const SolveConsts &c,
                                                   const float2 *__restrict__ wdk,
                                                   const float2 *__restrict__ e1k,
                                                   const float2 *__restrict__ e2k,
                                                   const float *__restrict__ e3k, bool inv,
                                                   float2 mu[3], float2 d[NT], float2 c6[6], float2 ec) {
  const Sym3d S = prior_d(c6, c.var0);
  float sf[6];
  prior_f(c6, c.var0, sf);
  // outside the band (or on failure) the reference keeps its float prior
  const int pa[6] = {0, 1, 2, 0, 0, 1}, pb[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
  for (int t = 0; t < 6; ++t) c6[t] = make_float2(sf[t], 0.f);
  if (!inv) return false;
  auto sgf = [&](int p, int q) -> float {
    if (p > q) { int t = p; p = q; q = t; }
    return p == 0 ? (q == 0 ? sf[0] : q == 1 ? sf[3] : sf[4]) : p == 1 ? (q == 1 ? sf[1] : sf[5]) : sf[2];
  };
  // AS = A S in FP64 (row l at AS[3 l .. 3 l + 2]), formed once
#pragma unroll
  for (int l = 0; l < NT; ++l)
#pragma unroll
    for (int p = 0; p < 3; ++p)
      AS[3 * l + p] = (double)c.A[l][0] * sget(S, 0, p) + (double)c.A[l][1] * sget(S, 1, p) +
                      (double)c.A[l][2] * sget(S, 2, p);
  {
    const double lam = fabs((double)ec.x);
    const double cc = 0.5 * (1.0 - (double)c.wnc) * lam;
    const float ccf = (float)cc;
#pragma unroll
    for (int l = 0; l < NT; ++l) {
      const double as0 = AS[3 * l], as1 = AS[3 * l + 1], as2 = AS[3 * l + 2];
      float af0 = 0.f, af1 = 0.f, af2 = 0.f;
#pragma unroll
      for (int r = 0; r < 3; ++r) {
        af0 += c.A[l][r] * sgf(r, 0);
        af1 += c.A[l][r] * sgf(r, 1);
        af2 += c.A[l][r] * sgf(r, 2);
      }
      const float2 wl = __ldg(wdk + l), e1l = __ldg(e1k + l), e2l = __ldg(e2k + l);
#pragma unroll
      for (int m = 0; m <= l; ++m) {
        const float2 wm = __ldg(wdk + m), e1m = __ldg(e1k + m), e2m = __ldg(e2k + m);
        const double th = c.theta[l][m];
        // FP64 copy
        {
          const double B = as0 * c.A[m][0] + as1 * c.A[m][1] + as2 * c.A[m][2];
          const double2 w = dmulc(make_double2(wl.x, wl.y), make_double2(wm.x, wm.y));
          const double2 n1 = dmulc(make_double2(e1l.x, e1l.y), make_double2(e1m.x, e1m.y));
          const double2 n2 = dmulc(make_double2(e2l.x, e2l.y), make_double2(e2m.x, e2m.y));
          const double f = cc * th;
          double2 v = make_double2(w.x * B + f * (n1.x + n2.x), w.y * B + f * (n1.y + n2.y));
          if (l == m) {
            const double e3 = (double)__ldg(e3k + l);
            v.x += (double)c.wnc * th * e3 * e3;
            v.y = 0.0;
          }
          Md[tri(l, m)] = v;
        }
        // FP32 build
        {
          const float B = af0 * c.A[m][0] + af1 * c.A[m][1] + af2 * c.A[m][2];
          const float2 w = cmulc(wl, wm), n1 = cmulc(e1l, e1m), n2 = cmulc(e2l, e2m);
          const float f = ccf * (float)th;
          float2 v = make_float2(w.x * B + f * (n1.x + n2.x), w.y * B + f * (n1.y + n2.y));
          if (l == m) {
            const float e3 = __ldg(e3k + l);
            v.x += c.wnc * (float)th * e3 * e3;
            v.y = 0.f;
          }
          Lf[tri(l, m)] = v;
        }
      }
    }
  }
  float rdf[NT];
  if (!cholesky<NT, float2, float, LAF>(Lf, rdf)) return true;
#pragma unroll
  for (int t = 0; t < 6; ++t) c6[t] = make_float2((float)sget(S, pa[t], pb[t]), 0.f);
  // residual of the prior mean, v = d - K mu (FP64), formed once
  double2 v[NT];
#pragma unroll
  for (int l = 0; l < NT; ++l) {
    double2 km = make_double2(0.0, 0.0);
#pragma unroll
    for (int r = 0; r < 3; ++r)
      km = dadd(km, make_double2(c.A[l][r] * (double)mu[r].x, c.A[l][r] * (double)mu[r].y));
    const float2 wl = __ldg(wdk + l);
    km = dmul(make_double2(wl.x, wl.y), km);
    v[l] = make_double2((double)d[l].x - km.x, (double)d[l].y - km.y);
  }
  double2 dm[3];  // mean corrections X^H v
  // rolled, as in the FP64 form
#pragma unroll 1
  for (int q = 0; q < 3; ++q) {
    double2 ks[NT];
    float2 x0[NT][3];  // column 0 used; solver works on [.][3] arrays
#pragma unroll
    for (int l = 0; l < NT; ++l) {
      const double as = AS[3 * l + q];
      const float2 wl = __ldg(wdk + l);
      ks[l] = make_double2(wl.x * as, wl.y * as);
      x0[l][0] = make_float2((float)ks[l].x, (float)ks[l].y);
    }
    // x0 = M^-1 ks (FP32), column 0 only
#pragma unroll
    for (int i = 0; i < NT; ++i) {
      float2 sacc = x0[i][0];
#pragma unroll
      for (int j = 0; j < i; ++j) {
        const float2 lij = Lf[tri(i, j)], xj = x0[j][0];
        sacc.x -= lij.x * xj.x - lij.y * xj.y;
        sacc.y -= lij.x * xj.y + lij.y * xj.x;
      }
      x0[i][0] = make_float2(sacc.x * rdf[i], sacc.y * rdf[i]);
    }
#pragma unroll
    for (int i = NT - 1; i >= 0; --i) {
      float2 sacc = x0[i][0];
#pragma unroll
      for (int j = i + 1; j < NT; ++j) {
        const float2 lji = Lf[tri(j, i)], xj = x0[j][0];
        sacc.x -= lji.x * xj.x + lji.y * xj.y;
        sacc.y -= lji.x * xj.y - lji.y * xj.x;
      }
      x0[i][0] = make_float2(sacc.x * rdf[i], sacc.y * rdf[i]);
    }
    // FP64 residual r = ks - Md x0, stored as the float right-hand side
#pragma unroll
    for (int l = 0; l < NT; ++l) {
      double2 acc = ks[l];
#pragma unroll
      for (int m = 0; m < NT; ++m) {
        const double2 Mlm = m <= l ? Md[tri(l, m)] : make_double2(Md[tri(m, l)].x, -Md[tri(m, l)].y);
        acc = dsub(acc, dmul(Mlm, make_double2(x0[m][0].x, x0[m][0].y)));
      }
      x0[l][1] = make_float2((float)acc.x, (float)acc.y);
    }
    // correction solve (FP32) on column 1
#pragma unroll
    for (int i = 0; i < NT; ++i) {
      float2 sacc = x0[i][1];
#pragma unroll
      for (int j = 0; j < i; ++j) {
        const float2 lij = Lf[tri(i, j)], xj = x0[j][1];
        sacc.x -= lij.x * xj.x - lij.y * xj.y;
        sacc.y -= lij.x * xj.y + lij.y * xj.x;
      }
      x0[i][1] = make_float2(sacc.x * rdf[i], sacc.y * rdf[i]);
    }
#pragma unroll
    for (int i = NT - 1; i >= 0; --i) {
      float2 sacc = x0[i][1];
#pragma unroll
      for (int j = i + 1; j < NT; ++j) {
        const float2 lji = Lf[tri(j, i)], xj = x0[j][1];
        sacc.x -= lji.x * xj.x + lji.y * xj.y;
        sacc.y -= lji.x * xj.y - lji.y * xj.x;
      }
      x0[i][1] = make_float2(sacc.x * rdf[i], sacc.y * rdf[i]);
    }
    double2 x[NT];
#pragma unroll
    for (int l = 0; l < NT; ++l)
      x[l] = make_double2((double)x0[l][0].x + (double)x0[l][1].x, (double)x0[l][0].y + (double)x0[l][1].y);
    // mean correction conj(x)^T v
    double2 acc = make_double2(0.0, 0.0);
#pragma unroll
    for (int l = 0; l < NT; ++l) acc = dadd(acc, dmulc(v[l], x[l]));
    if (q == 0) dm[0] = acc;
    else if (q == 1) dm[1] = acc;
    else dm[2] = acc;
    // FP64 Schur update of the entries (p, q), p <= q: S_pq - sum_l AS_lp u_l,
    // u = conj(w) x
#pragma unroll
    for (int l = 0; l < NT; ++l) {
      const float2 wl = __ldg(wdk + l);
      x[l] = make_double2(wl.x * x[l].x + wl.y * x[l].y, wl.x * x[l].y - wl.y * x[l].x);
    }
#pragma unroll
    for (int p = 0; p <= q; ++p) {
      double2 r = make_double2(0.0, 0.0);
#pragma unroll
      for (int l = 0; l < NT; ++l) {
        const double as = AS[3 * l + p];
        r.x += as * x[l].x;
        r.y += as * x[l].y;
      }
      const int t = p == q ? p : (p == 0 ? (q == 1 ? 3 : 4) : 5);
      c6[t] = make_float2((float)(sget(S, p, q) - r.x), (float)(-r.y));
    }
  }
  // residual d - K (mu + dm) = v - K dm; posterior mean mu + dm (FP64)
#pragma unroll
  for (int l = 0; l < NT; ++l) {
    double2 km = make_double2(0.0, 0.0);
#pragma unroll
    for (int r = 0; r < 3; ++r) km = dadd(km, make_double2(c.A[l][r] * dm[r].x, c.A[l][r] * dm[r].y));
    const float2 wl = __ldg(wdk + l);
    km = dmul(make_double2(wl.x, wl.y), km);
    d[l] = make_float2((float)(v[l].x - km.x), (float)(v[l].y - km.y));
  }
#pragma unroll
  for (int q = 0; q < 3; ++q)
    mu[q] = make_float2((float)((double)mu[q].x + dm[q].x), (float)((double)mu[q].y + dm[q].y));
  return false;
}

template <int NT>
__device__ __forceinline__ bool solve_bin_mixed(const SolveConsts &c, const float2 *__restrict__ wdk,
                                                const float2 *__restrict__ e1k,
                                                const float2 *__restrict__ e2k,
                                                const float *__restrict__ e3k, bool inv,
                                                float2 mu[3], float2 d[NT], float2 c6[6], float2 ec) {
  float2 Lf[NT * (NT + 1) / 2];
  double2 Md[NT * (NT + 1) / 2];
  double AS[3 * NT];
  return solve_bin_mixed_in<NT, float2 *, double2 *, double *>(Lf, Md, AS, c, wdk, e1k, e2k, e3k, inv, mu, d,
                                                               c6, ec);
}

// ---------------------------------------------------------------------------
// Square-root form of the per-bin update (FP64 and mixed forms of the
// standalone solve kernel).
//
// With M = L L^H, X = M^-1 K S and v = d - K mu, the reference's quantities
// (src/crava.cpp:1114-1129) are Gram products of forward substitutions only:
//   (K S)^H X = Y^H Y,   X^H v = Y^H z,   Y = L^-1 K S,  z = L^-1 v,
// so S_post = S - Y^H Y, mu_post = mu + Y^H z, r = d - K mu_post.  No back
// substitution and no X; the Schur subtraction stays in FP64 (the Gram
// product accumulates in FP64 in both forms).
//
// Per-kz constants (one kz plane per CTA, staged in shared memory): for the
// lower triangle (l, m <= l), W_lm = wd_l conj(wd_m) and
// E_lm = (1 - wnc)/2 theta_lm (e1_l conj(e1_m) + e2_l conj(e2_m)), and
// D_l = wnc theta_ll e3_l^2, so that per bin
//   M_lm = W_lm (A S A^T)_lm + lambda E_lm  (+ D_l on the diagonal),
// lambda = |Re(err spectrum)| (getNextErrorVariance, src/crava.cpp:1297-1334).
template <int NT>
struct KzConst {
  static constexpr int NP = NT * (NT + 1) / 2;
  double2 W[NP], E[NP];
  float2 Wf[NP], Ef[NP];
  double D[NT];
  float Df[NT];
  float2 wd[NT];
};

// Fills k for plane kz (call with every thread of the CTA, then sync).
template <int NT>
__device__ __forceinline__ void kz_const_fill(KzConst<NT> &k, const SolveConsts &c, const float2 *__restrict__ wdk,
                                              const float2 *__restrict__ e1k, const float2 *__restrict__ e2k,
                                              const float *__restrict__ e3k, int tid) {
  const double hw = 0.5 * (1.0 - (double)c.wnc);
  if (tid < KzConst<NT>::NP) {
    int l = 0;
    while (tri(l + 1, 0) <= tid) ++l;
    const int m = tid - tri(l, 0);
    const float2 wl = wdk[l], wm = wdk[m], al = e1k[l], am = e1k[m], bl = e2k[l], bm = e2k[m];
    const double2 w = dmulc(make_double2(wl.x, wl.y), make_double2(wm.x, wm.y));
    const double2 n1 = dmulc(make_double2(al.x, al.y), make_double2(am.x, am.y));
    const double2 n2 = dmulc(make_double2(bl.x, bl.y), make_double2(bm.x, bm.y));
    const double f = hw * c.theta[l][m];
    double2 e = make_double2(f * (n1.x + n2.x), f * (n1.y + n2.y));
    if (l == m) e.y = 0.0;
    k.W[tid] = l == m ? make_double2(w.x, 0.0) : w;
    k.E[tid] = e;
    const float2 wf = cmulc(wl, wm), n1f = cmulc(al, am), n2f = cmulc(bl, bm);
    const float ff = (float)f;
    k.Wf[tid] = l == m ? make_float2(wf.x, 0.f) : wf;
    k.Ef[tid] = make_float2(ff * (n1f.x + n2f.x), l == m ? 0.f : ff * (n1f.y + n2f.y));
  }
  if (tid < NT) {
    const double e3 = (double)e3k[tid];
    k.D[tid] = (double)c.wnc * c.theta[tid][tid] * e3 * e3;
    k.Df[tid] = (float)k.D[tid];
    k.wd[tid] = wdk[tid];
  }
}

// The prior in double: |Re(c)/S0| S0 (getNextParameterCovariance,
// src/seismicparametersholder.cpp:355-427) equals sign(S0) |Re(c)| exactly
// in double for float c (its rounding error is far below the float ulp),
// so it is formed without a division.
__device__ __forceinline__ Sym3d prior_exact(const float2 c6[6], const double v[6]) {
  double r[6];
#pragma unroll
  for (int t = 0; t < 6; ++t) {
    const double x = fabs((double)c6[t].x);
    r[t] = v[t] != 0.0 ? copysign(x, v[t]) : x;
  }
  return Sym3d{r[0], r[1], r[2], r[3], r[4], r[5]};
}

// (A S)_{l,p} for p = 0..2 in double.
template <typename T>
__device__ __forceinline__ void as_row(const SolveConsts &c, const Sym3d &S, int l, T as[3]) {
#pragma unroll
  for (int p = 0; p < 3; ++p)
    as[p] = (T)((double)c.A[l][0] * sget(S, 0, p) + (double)c.A[l][1] * sget(S, 1, p) +
                (double)c.A[l][2] * sget(S, 2, p));
}

// Cholesky of the square-root forms: as cholesky() (the reference's failure
// rules), but the reciprocal pivots 1 / L_ii are stored in the diagonal
// slots (the substitutions use nothing else of the diagonal), so they need
// no registers.
template <int NT, typename T2, typename T, typename LA>
__device__ __forceinline__ bool cholesky_rd(LA L) {
  const T factor = L[0].x;
  if (factor <= T(0)) return false;
  const T tol = (T)kTol * factor;
#pragma unroll
  for (int i = 0; i < NT; ++i) {
    if (L[tri(i, i)].x <= tol) return false;
#pragma unroll
    for (int j = 0; j < i; ++j) {
      T2 s = L[tri(i, j)];
#pragma unroll
      for (int k = 0; k < j; ++k) {
        const T2 a = L[tri(i, k)], b = L[tri(j, k)];
        s.x -= a.x * b.x + a.y * b.y;
        s.y -= a.y * b.x - a.x * b.y;
      }
      const T r = L[tri(j, j)].x;
      s.x *= r; s.y *= r;
      L[tri(i, j)] = s;
    }
    T d = L[tri(i, i)].x;
#pragma unroll
    for (int k = 0; k < i; ++k) d -= L[tri(i, k)].x * L[tri(i, k)].x + L[tri(i, k)].y * L[tri(i, k)].y;
    if (d <= tol) return false;
    L[tri(i, i)] = T2{rsqrt(d), T(0)};
  }
  return true;
}

// Forward substitution L x = b in place with 1 / L_ii in the diagonal slots.
template <int NT, typename T2, typename LA>
__device__ __forceinline__ void fwd_sub_rd(LA L, T2 *x) {
#pragma unroll
  for (int i = 0; i < NT; ++i) {
    T2 s = x[i];
#pragma unroll
    for (int j = 0; j < i; ++j) {
      const T2 lij = L[tri(i, j)], xj = x[j];
      s.x -= lij.x * xj.x - lij.y * xj.y;
      s.y -= lij.x * xj.y + lij.y * xj.x;
    }
    const auto r = L[tri(i, i)].x;
    x[i].x = s.x * r;
    x[i].y = s.y * r;
  }
}

// Back substitution L^H x = b in place with 1 / L_ii in the diagonal slots.
template <int NT, typename T2, typename LA>
__device__ __forceinline__ void bwd_sub_rd(LA L, T2 *x) {
#pragma unroll
  for (int i = NT - 1; i >= 0; --i) {
    T2 s = x[i];
#pragma unroll
    for (int j = i + 1; j < NT; ++j) {
      const T2 lji = L[tri(j, i)], xj = x[j];  // conj(lji) * xj
      s.x -= lji.x * xj.x + lji.y * xj.y;
      s.y -= lji.x * xj.y - lji.y * xj.x;
    }
    const auto r = L[tri(i, i)].x;
    x[i].x = s.x * r;
    x[i].y = s.y * r;
  }
}

// Where a bin's input spectra are read from: the grids themselves
// (GlobalIn) or a per-thread staging slot in shared memory filled
// asynchronously ahead of the computation (StagedIn: the inputs mu 0..2,
// data 0..NT-1, cov 0..5 and err, each entry STRIDE float2 apart).
struct GlobalIn {
  const SolveGrids *g;
  long long idx;
  __device__ __forceinline__ float2 mu(int q) const { return g->mu[q][idx]; }
  __device__ __forceinline__ float2 d(int l) const { return g->data[l][idx]; }
};
template <int NT, int STRIDE>
struct StagedIn {
  const float2 *s;
  __device__ __forceinline__ float2 mu(int q) const { return s[q * STRIDE]; }
  __device__ __forceinline__ float2 d(int l) const { return s[(3 + l) * STRIDE]; }
  __device__ __forceinline__ float2 cov(int t) const { return s[(3 + NT + t) * STRIDE]; }
  __device__ __forceinline__ float2 err() const { return s[(9 + NT) * STRIDE]; }
};

// v = d - K mu in double, from the bin's input spectra.
template <int NT, typename IN>
__device__ __forceinline__ void prior_resid_g(const SolveConsts &c, const KzConst<NT> &k, const IN &in,
                                              double2 v[NT]) {
  double2 m[3];
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    const float2 x = in.mu(r);
    m[r] = make_double2(x.x, x.y);
  }
#pragma unroll
  for (int l = 0; l < NT; ++l) {
    double2 km = make_double2(0.0, 0.0);
#pragma unroll
    for (int r = 0; r < 3; ++r) km = dadd(km, make_double2(c.A[l][r] * m[r].x, c.A[l][r] * m[r].y));
    const float2 wl = k.wd[l], dl = in.d(l);
    km = dmul(make_double2(wl.x, wl.y), km);
    v[l] = make_double2((double)dl.x - km.x, (double)dl.y - km.y);
  }
}

// Posterior mean mu + dm and residual d - K (mu + dm), written to the bin's
// spectra (the inputs re-read here, so they hold no registers during the
// solve).  Returns whether every output is finite.
template <int NT, typename IN>
__device__ __forceinline__ bool write_mean_resid(const SolveConsts &c, const KzConst<NT> &k, const SolveGrids &g,
                                                 long long idx, const IN &in, const double2 dm[3]) {
  double2 mp[3];
  bool ok = true;
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    const float2 x = in.mu(q);
    mp[q] = make_double2((double)x.x + dm[q].x, (double)x.y + dm[q].y);
  }
#pragma unroll
  for (int l = 0; l < NT; ++l) {
    double2 km = make_double2(0.0, 0.0);
#pragma unroll
    for (int r = 0; r < 3; ++r) km = dadd(km, make_double2(c.A[l][r] * mp[r].x, c.A[l][r] * mp[r].y));
    const float2 wl = k.wd[l], dl = in.d(l);
    km = dmul(make_double2(wl.x, wl.y), km);
    const float2 r = make_float2((float)((double)dl.x - km.x), (float)((double)dl.y - km.y));
    g.data[l][idx] = r;
    ok &= fin2(r);
  }
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    const float2 x = make_float2((float)mp[q].x, (float)mp[q].y);
    g.mu[q][idx] = x;
    ok &= fin2(x);
  }
  return ok;
}

// Posterior covariance entry (p, q) = S_pq - G_pq, written to its grid.
__device__ __forceinline__ bool write_cov(const SolveGrids &g, long long idx, int t, double s, double2 G) {
  const float2 x = make_float2((float)(s - G.x), t < 3 ? 0.f : (float)(-G.y));
  g.cov[t][idx] = x;
  return fin2(x);
}

// The G entries (p, q), p <= q, that column q of Y completes, in the order
// (0,0) (1,1) (2,2) (0,1) (0,2) (1,2).
__host__ __device__ constexpr int gidx(int p, int q) { return p == q ? p : (p == 0 ? (q == 1 ? 3 : 4) : 5); }

// Column q of K S: wd_l (A S)_lq.
template <int NT, typename T2>
__device__ __forceinline__ void ks_col(const SolveConsts &c, const KzConst<NT> &k, const Sym3d &S, int q, T2 y[NT]) {
#pragma unroll
  for (int l = 0; l < NT; ++l) {
    const double a = (double)c.A[l][0] * sget(S, 0, q) + (double)c.A[l][1] * sget(S, 1, q) +
                     (double)c.A[l][2] * sget(S, 2, q);
    const float2 wl = k.wd[l];
    y[l].x = wl.x * a;
    y[l].y = wl.y * a;
  }
}

// FP64 square-root form of one inverted bin, in place on the grids.  L:
// the FP64 factor (lower triangle, tri() indexing); Y: room for the first
// two columns of Y.  Returns false when the factorisation failed (then the
// caller writes the prior and keeps mu and the data).  *ok: every output
// finite.
template <int NT, typename LA, typename YA, typename IN>
__device__ __forceinline__ bool solve_bin_fp64_sq(LA L, YA Y, const SolveConsts &c, const KzConst<NT> &k,
                                                  const Sym3d &S, double lam, const SolveGrids &g, long long idx,
                                                  const IN &in, bool *ok) {
#pragma unroll
  for (int l = 0; l < NT; ++l) {
    double as[3];
    as_row(c, S, l, as);
#pragma unroll
    for (int m = 0; m <= l; ++m) {
      const double B = as[0] * c.A[m][0] + as[1] * c.A[m][1] + as[2] * c.A[m][2];
      const double2 w = k.W[tri(l, m)], e = k.E[tri(l, m)];
      double2 v = make_double2(w.x * B + lam * e.x, w.y * B + lam * e.y);
      if (l == m) { v.x += k.D[l]; v.y = 0.0; }
      L[tri(l, m)] = v;
    }
  }
  if (!cholesky_rd<NT, double2, double, LA>(L)) return false;
  // Y = L^-1 K S column by column; each column completes its Gram entries
  // (written at once) and the first two stay for the later columns
  bool fin = true;
  double2 y[NT];
#pragma unroll 1
  for (int q = 0; q < 3; ++q) {
    ks_col<NT, double2>(c, k, S, q, y);
    fwd_sub_rd<NT, double2, LA>(L, y);
    double2 gq = make_double2(0.0, 0.0), g0 = gq, g1 = gq;
#pragma unroll
    for (int l = 0; l < NT; ++l) {
      gq.x += y[l].x * y[l].x + y[l].y * y[l].y;
      if (q >= 1) g0 = dadd(g0, dmulc(y[l], Y[l]));       // conj(y0) y
      if (q >= 2) g1 = dadd(g1, dmulc(y[l], Y[NT + l]));  // conj(y1) y
      if (q < 2) Y[q * NT + l] = y[l];
    }
    fin &= write_cov(g, idx, q, sget(S, q, q), gq);
    if (q >= 1) fin &= write_cov(g, idx, gidx(0, q), sget(S, 0, q), g0);
    if (q >= 2) fin &= write_cov(g, idx, gidx(1, q), sget(S, 1, q), g1);
  }
  // mean correction Y^H z, z = L^-1 (d - K mu); y holds the last column
  double2 z[NT];
  prior_resid_g<NT>(c, k, in, z);
  fwd_sub_rd<NT, double2, LA>(L, z);
  double2 dm[3] = {make_double2(0.0, 0.0), make_double2(0.0, 0.0), make_double2(0.0, 0.0)};
#pragma unroll
  for (int l = 0; l < NT; ++l) {
    dm[0] = dadd(dm[0], dmulc(z[l], Y[l]));
    dm[1] = dadd(dm[1], dmulc(z[l], Y[NT + l]));
    dm[2] = dadd(dm[2], dmulc(z[l], y[l]));
  }
  fin &= write_mean_resid<NT>(c, k, g, idx, in, dm);
  *ok = fin;
  return true;
}

// Mixed form of one inverted bin: M built and factorised in FP32, Y and z
// by FP32 forward substitution, the Gram products and the Schur
// subtraction in FP64.  A bin whose FP32 factor is ill-conditioned --
// (max L_ii / min L_ii)^2, a lower bound of cond(M), above kappa_refine --
// instead takes one step of FP64 iterative refinement on X = M^-1 K S: X0
// from the FP32 factor, the residual K S - M X0 in FP64 (M re-formed in
// FP64 from the per-kz constants), X = X0 + M^-1 r with the FP32 factor,
// then S_post = S - (K S)^H X and mu_post = mu + X^H v in FP64.  Lf: the
// FP32 factor; Yf: two FP32 columns; V: the FP64 prior-mean residual.
// Returns false when the FP32 factorisation failed.
template <int NT, typename LA, typename YA, typename VA, typename IN>
__device__ __forceinline__ bool solve_bin_mixed_sq(LA Lf, YA Yf, VA V, const SolveConsts &c, const KzConst<NT> &k,
                                                   const Sym3d &S, float kappa_refine, float lamf, double lam,
                                                   const SolveGrids &g, long long idx, const IN &in, bool *ok,
                                                   bool *refined) {
#pragma unroll
  for (int l = 0; l < NT; ++l) {
    float as[3];
    as_row(c, S, l, as);
#pragma unroll
    for (int m = 0; m <= l; ++m) {
      const float B = as[0] * c.A[m][0] + as[1] * c.A[m][1] + as[2] * c.A[m][2];
      const float2 w = k.Wf[tri(l, m)], e = k.Ef[tri(l, m)];
      float2 v = make_float2(w.x * B + lamf * e.x, w.y * B + lamf * e.y);
      if (l == m) { v.x += k.Df[l]; v.y = 0.f; }
      Lf[tri(l, m)] = v;
    }
  }
  if (!cholesky_rd<NT, float2, float, LA>(Lf)) return false;
  // diagonal slots hold 1 / L_ii: cond bound (max L_ii / min L_ii)^2
  float rmax = 0.f, rmin = 3.0e38f;
#pragma unroll
  for (int i = 0; i < NT; ++i) {
    const float r = Lf[tri(i, i)].x;
    rmax = fmaxf(rmax, r);
    rmin = fminf(rmin, r);
  }
  const float ratio = rmax / rmin;
  double2 dm[3];
  bool fin = true;
  *refined = ratio * ratio > kappa_refine;
  if (!*refined) {
    float2 y[NT];
#pragma unroll 1
    for (int q = 0; q < 3; ++q) {
      ks_col<NT, float2>(c, k, S, q, y);
      fwd_sub_rd<NT, float2, LA>(Lf, y);
      double2 gq = make_double2(0.0, 0.0), g0 = gq, g1 = gq;
#pragma unroll
      for (int l = 0; l < NT; ++l) {
        const double2 yl = make_double2(y[l].x, y[l].y);
        gq.x += yl.x * yl.x + yl.y * yl.y;
        if (q >= 1) { const float2 t = Yf[l]; g0 = dadd(g0, dmulc(yl, make_double2(t.x, t.y))); }
        if (q >= 2) { const float2 t = Yf[NT + l]; g1 = dadd(g1, dmulc(yl, make_double2(t.x, t.y))); }
        if (q < 2) Yf[q * NT + l] = y[l];
      }
      fin &= write_cov(g, idx, q, sget(S, q, q), gq);
      if (q >= 1) fin &= write_cov(g, idx, gidx(0, q), sget(S, 0, q), g0);
      if (q >= 2) fin &= write_cov(g, idx, gidx(1, q), sget(S, 1, q), g1);
    }
    float2 z[NT];
    {
      double2 v[NT];
      prior_resid_g<NT>(c, k, in, v);
#pragma unroll
      for (int l = 0; l < NT; ++l) z[l] = make_float2((float)v[l].x, (float)v[l].y);
    }
    fwd_sub_rd<NT, float2, LA>(Lf, z);
    dm[0] = dm[1] = dm[2] = make_double2(0.0, 0.0);
#pragma unroll
    for (int l = 0; l < NT; ++l) {
      const double2 zl = make_double2(z[l].x, z[l].y);
      const float2 y0 = Yf[l], y1 = Yf[NT + l];
      dm[0] = dadd(dm[0], dmulc(zl, make_double2(y0.x, y0.y)));
      dm[1] = dadd(dm[1], dmulc(zl, make_double2(y1.x, y1.y)));
      dm[2] = dadd(dm[2], dmulc(zl, make_double2(y[l].x, y[l].y)));
    }
  } else {
    {
      double2 v[NT];
      prior_resid_g<NT>(c, k, in, v);
#pragma unroll
      for (int l = 0; l < NT; ++l) V[l] = v[l];
    }
#pragma unroll 1
    for (int q = 0; q < 3; ++q) {
      float2 x0[NT], r[NT];
      {
        double2 ks[NT];
        ks_col<NT, double2>(c, k, S, q, ks);
#pragma unroll
        for (int l = 0; l < NT; ++l) x0[l] = make_float2((float)ks[l].x, (float)ks[l].y);
        fwd_sub_rd<NT, float2, LA>(Lf, x0);
        bwd_sub_rd<NT, float2, LA>(Lf, x0);
        // r = ks - M x0 in FP64, M_lm = W_lm B_lm + lambda E_lm (+ D_l)
#pragma unroll
        for (int l = 0; l < NT; ++l) {
          double asl[3];
          as_row(c, S, l, asl);
          double2 acc = ks[l];
#pragma unroll
          for (int m = 0; m < NT; ++m) {
            const int lo = l >= m ? l : m, hi = l >= m ? m : l;
            const double B = asl[0] * c.A[m][0] + asl[1] * c.A[m][1] + asl[2] * c.A[m][2];
            const double2 w = k.W[tri(lo, hi)], e = k.E[tri(lo, hi)];
            double2 Mlm = make_double2(w.x * B + lam * e.x, w.y * B + lam * e.y);
            if (l < m) Mlm.y = -Mlm.y;  // upper triangle: conj of the stored lower entry
            if (l == m) { Mlm.x += k.D[l]; Mlm.y = 0.0; }
            acc = dsub(acc, dmul(Mlm, make_double2(x0[m].x, x0[m].y)));
          }
          r[l] = make_float2((float)acc.x, (float)acc.y);
        }
      }
      fwd_sub_rd<NT, float2, LA>(Lf, r);
      bwd_sub_rd<NT, float2, LA>(Lf, r);
      double2 x[NT];
#pragma unroll
      for (int l = 0; l < NT; ++l) x[l] = make_double2((double)x0[l].x + (double)r[l].x, (double)x0[l].y + (double)r[l].y);
      double2 acc = make_double2(0.0, 0.0);
#pragma unroll
      for (int l = 0; l < NT; ++l) acc = dadd(acc, dmulc(V[l], x[l]));  // conj(x) v
      if (q == 0) dm[0] = acc;
      else if (q == 1) dm[1] = acc;
      else dm[2] = acc;
      // (K S)^H X entries (p, q), p <= q: sum_l AS_lp conj(w_l) x_l
#pragma unroll
      for (int l = 0; l < NT; ++l) {
        const float2 wl = k.wd[l];
        x[l] = make_double2(wl.x * x[l].x + wl.y * x[l].y, wl.x * x[l].y - wl.y * x[l].x);
      }
#pragma unroll
      for (int p = 0; p <= q; ++p) {
        double2 gg = make_double2(0.0, 0.0);
#pragma unroll
        for (int l = 0; l < NT; ++l) {
          double as[3];
          as_row(c, S, l, as);
          const double a = p == 0 ? as[0] : p == 1 ? as[1] : as[2];
          gg.x += a * x[l].x;
          gg.y += a * x[l].y;
        }
        fin &= write_cov(g, idx, gidx(p, q), sget(S, p, q), gg);
      }
    }
  }
  fin &= write_mean_resid<NT>(c, k, g, idx, in, dm);
  *ok = fin;
  return true;
}

// A band-gated bin: only the prior covariance is written (mu and the data
// stay as they are), in the arithmetic of the PREC form.
template <int PREC>
__device__ __forceinline__ void prior_only(const SolveConsts &c, float2 c6[6]) {
  if (PREC == 0) {
    const Sym3d S = prior_d(c6, c.var0);
    const int pa[6] = {0, 1, 2, 0, 0, 1}, pb[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
    for (int t = 0; t < 6; ++t) c6[t] = make_float2((float)sget(S, pa[t], pb[t]), 0.f);
  } else {
    float sf[6];
    prior_f(c6, c.var0, sf);
#pragma unroll
    for (int t = 0; t < 6; ++t) c6[t] = make_float2(sf[t], 0.f);
  }
}

// One bin.  In: mu[3], d[NT], c6[6] (the six prior spectra), ec (noise
// correlation spectrum), the bin's kz tables and its band flag.  Out (in
// place): mu <- posterior mean, d <- residual, c6 <- posterior covariance
// (0,0) (1,1) (2,2) (0,1) (0,2) (1,2).  Returns true when an inverted bin's
// factorisation failed (the prior is kept, as src/crava.cpp:1109-1111).
// PREC 0: FP64 throughout.  PREC 1: FP32 build and factorisation, one FP64
// refinement step on the residual K S - M X0, FP64 Schur update and mean.
template <int NT, int PREC>
__device__ __forceinline__ bool solve_bin(const SolveConsts &c, const float2 *__restrict__ wdk,
                                          const float2 *__restrict__ e1k,
                                          const float2 *__restrict__ e2k,
                                          const float *__restrict__ e3k, bool inv,
                                          float2 mu[3], float2 d[NT], float2 c6[6], float2 ec) {
  if (PREC == 0) return solve_bin_fp64<NT>(c, wdk, e1k, e2k, e3k, inv, mu, d, c6, ec);
  if (PREC == 1) return solve_bin_mixed<NT>(c, wdk, e1k, e2k, e3k, inv, mu, d, c6, ec);
  float2 out_mu[3], out_r[NT];
  const Sym3d S = prior_d(c6, c.var0);
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
#pragma unroll
  for (int q = 0; q < 3; ++q) mu[q] = out_mu[q];
#pragma unroll
  for (int l = 0; l < NT; ++l) d[l] = out_r[l];
#pragma unroll
  for (int t = 0; t < 6; ++t) c6[t] = make_float2((float)Sp[t].x, (float)Sp[t].y);
  return fail;
}

}  // namespace sb
}  // namespace crava
