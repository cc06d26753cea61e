// woodbury.cuh -- the FP64 per-bin posterior through the noise-whitened
// (Woodbury) form.
//
// The reference forms M = K S K^H + N per inverted bin and factors it
// (src/crava.cpp:1104-1130): a 5x5 complex Cholesky at five angles.  N is
// the noise covariance, N = lambda E + Dg: E (the angle-correlated part,
// (1 - wnc)/2 theta_lm (e1_l conj(e1_m) + e2_l conj(e2_m))) and the
// diagonal Dg (wnc theta_ll e3_l^2) depend on the kz plane only, lambda =
// |Re(err spectrum)| on the bin (src/crava.cpp:1297-1334).  With the
// eigendecomposition Dg^{-1/2} E Dg^{-1/2} = V diag(m) V^H of the plane,
//   N = Dg^{1/2} V (lambda diag(m) + I) V^H Dg^{1/2},
//   N^-1 = T^H diag(c) T,  T = V^H Dg^{-1/2},  c_i = 1 / (lambda m_i + 1),
// so per bin only the nt scalars c_i vary.  With W = T K (nt x 3, per
// plane) the posterior is
//   P = K^H N^-1 K = W^H diag(c) W                     (3x3 Hermitian)
//   S_post = (S^-1 + P)^-1 = Z^H Z,  Z = R^-1 LS^T,
//       S = LS LS^T (real Cholesky of the prior), I + LS^T P LS = R R^H
//   mu_post = mu + S_post W^H diag(c) T (d - K mu)
// -- the same quantities as S - (KS)^H M^-1 KS and mu + (KS)^H M^-1 (d -
// K mu), with 3x3 instead of nt x nt factorisations, no cancellation in the
// covariance (a Gram product), and I + LS^T P LS has every eigenvalue >= 1.
// About 600 FP64 operations per bin at five angles against about 1400 for
// the square-root form of M, and far fewer live registers.
//
// Where the form does not apply the bin goes to the square-root form of M,
// which keeps the reference's failure rules: a plane whose Dg has a zero
// (or whose eigendecomposition did not converge), and a bin whose prior S
// is not positive definite or whose lambda m_i + 1 is not positive (or not
// finite).  For every other bin M = K S K^H + N is positive definite, so
// the reference's Cholesky succeeds and the results agree to rounding.
#pragma once

#include <math.h>

#include "solve_bin.cuh"

namespace crava {
namespace sb {

// Per-plane constants of the Woodbury form (CRAVA_GPU_MAX_THETA = 8).
struct WbTable {
  double2 T[8][8];  // V^H Dg^{-1/2}: t = T r
  double2 W[8][3];  // T K
  // per eigen-direction i, the terms of P = sum_i c_i conj(W_i)^T W_i:
  // |W_i0|^2 |W_i1|^2 |W_i2|^2, conj(W_i0) W_i1, conj(W_i0) W_i2,
  // conj(W_i1) W_i2 (re, im)
  double H[8][9];
  double m[8];      // eigenvalues of Dg^{-1/2} E Dg^{-1/2}
  int ok;           // the plane can use the form
  int pad[3];
};

__host__ __device__ __forceinline__ double2 d2(double x, double y) { return make_double2(x, y); }
__host__ __device__ __forceinline__ double2 dconj(double2 a) { return d2(a.x, -a.y); }
__host__ __device__ __forceinline__ double2 dcm(double2 a, double2 b) {  // a * b
  return d2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ double2 dcmc(double2 a, double2 b) {  // conj(a) * b
  return d2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}

// Cyclic Jacobi eigendecomposition of a Hermitian NT x NT matrix: a <-
// diag(m), v unitary with A v = v diag(m).  Each rotation first turns
// a_pq real by a phase on column q, then applies the real 2x2 Jacobi
// rotation with tan 2th = 2 |a_pq| / (a_qq - a_pp).  Returns false if the
// off-diagonal mass did not fall below 1e-32 of the matrix's in 50 sweeps.
template <int NT>
__host__ __device__ inline bool herm_jacobi(double2 (&a)[NT][NT], double2 (&v)[NT][NT], double (&m)[NT]) {
  double scale = 0.0;
  for (int i = 0; i < NT; ++i)
    for (int j = 0; j < NT; ++j) {
      v[i][j] = d2(i == j ? 1.0 : 0.0, 0.0);
      scale += a[i][j].x * a[i][j].x + a[i][j].y * a[i][j].y;
    }
  bool conv = false;
  for (int sweep = 0; sweep < 50 && !conv; ++sweep) {
    double off = 0.0;
    for (int p = 0; p < NT; ++p)
      for (int q = p + 1; q < NT; ++q) off += a[p][q].x * a[p][q].x + a[p][q].y * a[p][q].y;
    if (off <= 1e-32 * scale) {
      conv = true;
      break;
    }
    for (int p = 0; p < NT; ++p)
      for (int q = p + 1; q < NT; ++q) {
        const double mag = hypot(a[p][q].x, a[p][q].y);
        if (mag == 0.0) continue;
        const double2 e = d2(a[p][q].x / mag, a[p][q].y / mag);
        const double th = 0.5 * atan2(2.0 * mag, a[q][q].x - a[p][p].x);
        const double c = cos(th), s = sin(th);
        const double2 se = d2(s * e.x, s * e.y), sec = dconj(se);  // s e, s conj(e)
        const double2 ce = d2(c * e.x, c * e.y), cec = dconj(ce);
        for (int i = 0; i < NT; ++i) {  // columns: A <- A J
          const double2 x = a[i][p], y = a[i][q];
          const double2 ys = dcm(sec, y), yc = dcm(cec, y);
          a[i][p] = d2(c * x.x - ys.x, c * x.y - ys.y);
          a[i][q] = d2(s * x.x + yc.x, s * x.y + yc.y);
        }
        for (int j = 0; j < NT; ++j) {  // rows: A <- J^H A
          const double2 x = a[p][j], y = a[q][j];
          const double2 ys = dcm(se, y), yc = dcm(ce, y);
          a[p][j] = d2(c * x.x - ys.x, c * x.y - ys.y);
          a[q][j] = d2(s * x.x + yc.x, s * x.y + yc.y);
        }
        for (int i = 0; i < NT; ++i) {  // V <- V J
          const double2 x = v[i][p], y = v[i][q];
          const double2 ys = dcm(sec, y), yc = dcm(cec, y);
          v[i][p] = d2(c * x.x - ys.x, c * x.y - ys.y);
          v[i][q] = d2(s * x.x + yc.x, s * x.y + yc.y);
        }
        a[p][q] = a[q][p] = d2(0.0, 0.0);
        a[p][p].y = 0.0;
        a[q][q].y = 0.0;
      }
  }
  for (int i = 0; i < NT; ++i) m[i] = a[i][i].x;
  return conv;
}

// The plane's table from its kz tables (wd, e1, e2, e3: nt entries each)
// and the solve constants; E and Dg exactly as kz_const_fill forms them.
template <int NT>
__host__ __device__ inline void wb_table_fill(WbTable &w, const SolveConsts &c, const float2 *wdk, const float2 *e1k,
                                              const float2 *e2k, const float *e3k) {
  const double hw = 0.5 * (1.0 - (double)c.wnc);
  double dg[NT], rs[NT];
  bool ok = true;
  for (int l = 0; l < NT; ++l) {
    const double e3 = (double)e3k[l];
    dg[l] = (double)c.wnc * c.theta[l][l] * e3 * e3;
    ok = ok && dg[l] > 0.0 && dg[l] < 1e300;
    rs[l] = ok ? 1.0 / sqrt(dg[l]) : 0.0;
  }
  double2 a[NT][NT], v[NT][NT];
  double m[NT];
  for (int l = 0; l < NT; ++l)
    for (int k = 0; k < NT; ++k) {
      const double2 al = d2(e1k[l].x, e1k[l].y), ak = d2(e1k[k].x, e1k[k].y);
      const double2 bl = d2(e2k[l].x, e2k[l].y), bk = d2(e2k[k].x, e2k[k].y);
      const double2 n1 = dcmc(ak, al), n2 = dcmc(bk, bl);  // e1_l conj(e1_k), e2_l conj(e2_k)
      const double f = hw * c.theta[l][k] * rs[l] * rs[k];
      a[l][k] = d2(f * (n1.x + n2.x), l == k ? 0.0 : f * (n1.y + n2.y));
    }
  ok = ok && herm_jacobi<NT>(a, v, m);
  for (int i = 0; i < 8; ++i) {
    for (int l = 0; l < 8; ++l) w.T[i][l] = d2(0.0, 0.0);
    for (int p = 0; p < 3; ++p) w.W[i][p] = d2(0.0, 0.0);
    for (int t = 0; t < 9; ++t) w.H[i][t] = 0.0;
    w.m[i] = 0.0;
  }
  for (int i = 0; i < NT; ++i) {
    ok = ok && isfinite(m[i]);
    w.m[i] = m[i];
    for (int l = 0; l < NT; ++l) w.T[i][l] = d2(v[l][i].x * rs[l], -v[l][i].y * rs[l]);  // conj(V_li) / sqrt(Dg_l)
    double2 W3[3];
    for (int p = 0; p < 3; ++p) {
      double2 s = d2(0.0, 0.0);
      for (int l = 0; l < NT; ++l) {
        const double2 kl = d2(c.A[l][p] * (double)wdk[l].x, c.A[l][p] * (double)wdk[l].y);  // K_lp = wd_l A_lp
        const double2 t = dcm(w.T[i][l], kl);
        s = d2(s.x + t.x, s.y + t.y);
      }
      W3[p] = s;
      w.W[i][p] = s;
    }
    w.H[i][0] = W3[0].x * W3[0].x + W3[0].y * W3[0].y;
    w.H[i][1] = W3[1].x * W3[1].x + W3[1].y * W3[1].y;
    w.H[i][2] = W3[2].x * W3[2].x + W3[2].y * W3[2].y;
    const double2 h01 = dcmc(W3[0], W3[1]), h02 = dcmc(W3[0], W3[2]), h12 = dcmc(W3[1], W3[2]);
    w.H[i][3] = h01.x; w.H[i][4] = h01.y;
    w.H[i][5] = h02.x; w.H[i][6] = h02.y;
    w.H[i][7] = h12.x; w.H[i][8] = h12.y;
  }
  w.ok = ok ? 1 : 0;
  w.pad[0] = w.pad[1] = w.pad[2] = 0;
}

// Real Cholesky of the 3x3 prior, LS = [l0 0 0; l1 l2 0; l3 l4 l5].
// Returns false unless every pivot is positive (a NaN fails too).
__device__ __forceinline__ bool chol3(const Sym3d &S, double (&L)[6]) {
  const double p0 = sget(S, 0, 0);
  if (!(p0 > 0.0)) return false;
  L[0] = sqrt(p0);
  const double r0 = 1.0 / L[0];
  L[1] = sget(S, 0, 1) * r0;
  L[3] = sget(S, 0, 2) * r0;
  const double p1 = sget(S, 1, 1) - L[1] * L[1];
  if (!(p1 > 0.0)) return false;
  L[2] = sqrt(p1);
  L[4] = (sget(S, 1, 2) - L[3] * L[1]) / L[2];
  const double p2 = sget(S, 2, 2) - L[3] * L[3] - L[4] * L[4];
  if (!(p2 > 0.0)) return false;
  L[5] = sqrt(p2);
  return true;
}

// The per-bin factors c_i = 1 / (lambda m_i + 1); false unless every
// lambda m_i + 1 is positive and finite.
template <int NT>
__device__ __forceinline__ bool wb_weights(const WbTable &w, double lam, double (&cw)[NT]) {
  bool ok = true;
#pragma unroll
  for (int i = 0; i < NT; ++i) {
    const double den = lam * w.m[i] + 1.0;
    ok = ok && den > 0.0 && den < 1e300;
    cw[i] = 1.0 / den;
  }
  return ok;
}

// One inverted bin in the Woodbury form, in place on the grids (the caller
// has checked chol3 and wb_weights).  Returns whether every output is
// finite.
template <int NT, typename IN>
__device__ __forceinline__ bool solve_bin_wb(const WbTable &w, const SolveConsts &c, const float2 *wd,
                                             const double (&L)[6], const double (&cw)[NT], const SolveGrids &g,
                                             long long idx, const IN &in) {
  // g = W^H diag(c) T (d - K mu)
  double2 gv[3] = {d2(0.0, 0.0), d2(0.0, 0.0), d2(0.0, 0.0)};
  {
    double2 r[NT];
    double2 m[3];
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const float2 x = in.mu(q);
      m[q] = d2(x.x, x.y);
    }
#pragma unroll
    for (int l = 0; l < NT; ++l) {
      double2 km = d2(0.0, 0.0);
#pragma unroll
      for (int q = 0; q < 3; ++q) km = d2(km.x + c.A[l][q] * m[q].x, km.y + c.A[l][q] * m[q].y);
      km = dcm(d2(wd[l].x, wd[l].y), km);
      const float2 dl = in.d(l);
      r[l] = d2((double)dl.x - km.x, (double)dl.y - km.y);
    }
#pragma unroll
    for (int i = 0; i < NT; ++i) {
      double2 t = d2(0.0, 0.0);
#pragma unroll
      for (int l = 0; l < NT; ++l) {
        const double2 x = dcm(w.T[i][l], r[l]);
        t = d2(t.x + x.x, t.y + x.y);
      }
      t = d2(cw[i] * t.x, cw[i] * t.y);
#pragma unroll
      for (int p = 0; p < 3; ++p) {
        const double2 x = dcmc(w.W[i][p], t);
        gv[p] = d2(gv[p].x + x.x, gv[p].y + x.y);
      }
    }
  }
  // P = sum_i c_i H_i (diagonal real, off-diagonal (p, q) = conj-row p x row q)
  double P[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
  for (int i = 0; i < NT; ++i)
#pragma unroll
    for (int t = 0; t < 9; ++t) P[t] += cw[i] * w.H[i][t];
  const double2 P01 = d2(P[3], P[4]), P02 = d2(P[5], P[6]), P12 = d2(P[7], P[8]);
  // X = P LS (LS lower triangular real), then Q = LS^T X (Hermitian; the
  // lower triangle and the diagonal are used)
  const double l0 = L[0], l1 = L[1], l2 = L[2], l3 = L[3], l4 = L[4], l5 = L[5];
  // column j of LS: (l0, l1, l3), (0, l2, l4), (0, 0, l5); P row p
  // P = [P0 P01 P02; conj(P01) P1 P12; conj(P02) conj(P12) P2]
  const double2 X00 = d2(P[0] * l0 + P01.x * l1 + P02.x * l3, P01.y * l1 + P02.y * l3);
  const double2 X10 = d2(P01.x * l0 + P[1] * l1 + P12.x * l3, -P01.y * l0 + P12.y * l3);
  const double2 X20 = d2(P02.x * l0 + P12.x * l1 + P[2] * l3, -P02.y * l0 - P12.y * l1);
  const double2 X11 = d2(P[1] * l2 + P12.x * l4, P12.y * l4);
  const double2 X21 = d2(P12.x * l2 + P[2] * l4, -P12.y * l2);
  const double X22 = P[2] * l5;
  // Q = LS^T X: rows of LS^T are (l0, l1, l3), (0, l2, l4), (0, 0, l5)
  const double Q00 = l0 * X00.x + l1 * X10.x + l3 * X20.x;
  const double2 Q10 = d2(l2 * X10.x + l4 * X20.x, l2 * X10.y + l4 * X20.y);
  const double2 Q20 = d2(l5 * X20.x, l5 * X20.y);
  const double Q11 = l2 * X11.x + l4 * X21.x;
  const double2 Q21 = d2(l5 * X21.x, l5 * X21.y);
  const double Q22 = l5 * X22;
  // R R^H = I + Q (every eigenvalue >= 1)
  const double r00 = sqrt(1.0 + Q00), i00 = 1.0 / r00;
  const double2 r10 = d2(Q10.x * i00, Q10.y * i00), r20 = d2(Q20.x * i00, Q20.y * i00);
  const double r11 = sqrt(1.0 + Q11 - (r10.x * r10.x + r10.y * r10.y)), i11 = 1.0 / r11;
  const double2 q21 = dcm(r20, dconj(r10));
  const double2 r21 = d2((Q21.x - q21.x) * i11, (Q21.y - q21.y) * i11);
  const double r22 = sqrt(1.0 + Q22 - (r20.x * r20.x + r20.y * r20.y) - (r21.x * r21.x + r21.y * r21.y));
  const double i22 = 1.0 / r22;
  // Z = R^-1 LS^T, column by column (column j of LS^T = row j of LS)
  double2 Z[3][3];
  const double b[3][3] = {{l0, 0.0, 0.0}, {l1, l2, 0.0}, {l3, l4, l5}};  // b[j] = column j of LS^T
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    const double2 z0 = d2(b[j][0] * i00, 0.0);
    const double2 t1 = dcm(r10, z0);
    const double2 z1 = d2((b[j][1] - t1.x) * i11, -t1.y * i11);
    const double2 t2 = dcm(r20, z0), t3 = dcm(r21, z1);
    const double2 z2 = d2((b[j][2] - t2.x - t3.x) * i22, (-t2.y - t3.y) * i22);
    Z[0][j] = z0; Z[1][j] = z1; Z[2][j] = z2;
  }
  // S_post = Z^H Z, mu_post = mu + S_post g
  double2 Sp[3][3];
#pragma unroll
  for (int p = 0; p < 3; ++p)
#pragma unroll
    for (int q = p; q < 3; ++q) {
      double2 s = d2(0.0, 0.0);
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const double2 x = dcmc(Z[k][p], Z[k][q]);
        s = d2(s.x + x.x, s.y + x.y);
      }
      Sp[p][q] = s;
      Sp[q][p] = dconj(s);
    }
  bool fin = true;
  const int tp[6] = {0, 1, 2, 0, 0, 1}, tq[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
  for (int t = 0; t < 6; ++t) {
    const double2 s = Sp[tp[t]][tq[t]];
    const float2 x = make_float2((float)s.x, t < 3 ? 0.f : (float)s.y);
    g.cov[t][idx] = x;
    fin &= fin2(x);
  }
  double2 dm[3];
#pragma unroll
  for (int p = 0; p < 3; ++p) {
    double2 s = d2(0.0, 0.0);
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const double2 x = dcm(Sp[p][q], gv[q]);
      s = d2(s.x + x.x, s.y + x.y);
    }
    dm[p] = s;
  }
  double2 mp[3];
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    const float2 x = in.mu(q);
    mp[q] = d2((double)x.x + dm[q].x, (double)x.y + dm[q].y);
  }
#pragma unroll
  for (int l = 0; l < NT; ++l) {
    double2 km = d2(0.0, 0.0);
#pragma unroll
    for (int q = 0; q < 3; ++q) km = d2(km.x + c.A[l][q] * mp[q].x, km.y + c.A[l][q] * mp[q].y);
    km = dcm(d2(wd[l].x, wd[l].y), km);
    const float2 dl = in.d(l);
    const float2 r = make_float2((float)((double)dl.x - km.x), (float)((double)dl.y - km.y));
    g.data[l][idx] = r;
    fin &= fin2(r);
  }
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    const float2 x = make_float2((float)mp[q].x, (float)mp[q].y);
    g.mu[q][idx] = x;
    fin &= fin2(x);
  }
  return fin;
}

}  // namespace sb
}  // namespace crava
