// lib_matr_ref.cuh -- device restatements of the reference's complex
// Cholesky factorisation and substitution, in its float operations and
// order: lib_matrCholCpx (libs/lib/lib_matr.c:78-167) and
// lib_matrAXeqBMatCpx (:330-365).  Files that include this header are
// compiled with -fmad=false, so each float operation rounds once, as in
// the reference's x86 build, and the results equal the reference's bit for
// bit.
#pragma once

namespace crava {

// lib_matrCholCpx on the lower triangle of m (normalised by m[0][0] first,
// rescaled at the end).  Returns 0 on success, 1 where the reference's
// factorisation reports failure.
template <int NT>
__device__ __forceinline__ int chol_ref(float2 (*m)[NT]) {
  float2 lr;
  float help;
  float factor = m[0][0].x;
  if (factor <= 0) return 1;
#pragma unroll
  for (int i = 0; i < NT; ++i)
#pragma unroll
    for (int j = 0; j < NT; ++j) { m[i][j].x = m[i][j].x / factor; m[i][j].y = m[i][j].y / factor; }
#pragma unroll
  for (int i = 0; i < NT; ++i) {
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
  for (int i = 0; i < NT; ++i)
#pragma unroll
    for (int j = 0; j <= i; ++j) { m[i][j].x *= sf; m[i][j].y *= sf; }
  return 0;
}

// lib_matrAXeqBMatCpx: solves L L^H X = B for the NC columns of B in place
// (forward then backward substitution, column by column).
template <int NT, int NC>
__device__ __forceinline__ void axeqb_ref(float2 (*L)[NT], float2 (*B)[NC]) {
  float2 lx;
  float help;
#pragma unroll
  for (int c = 0; c < NC; ++c) {
#pragma unroll
    for (int i = 0; i < NT; ++i) {
      lx = B[i][c];
#pragma unroll
      for (int j = 0; j < i; ++j) {
        lx.x -= (B[j][c].x * L[i][j].x - B[j][c].y * L[i][j].y);
        lx.y -= (B[j][c].y * L[i][j].x + B[j][c].x * L[i][j].y);
      }
      help = (L[i][i].x * L[i][i].x + L[i][i].y * L[i][i].y);
      B[i][c].x = (lx.x * L[i][i].x + lx.y * L[i][i].y) / help;
      B[i][c].y = (lx.y * L[i][i].x - lx.x * L[i][i].y) / help;
    }
#pragma unroll
    for (int i = NT - 1; i >= 0; --i) {
      lx = B[i][c];
#pragma unroll
      for (int j = NT - 1; j > i; --j) {
        lx.x = lx.x - (B[j][c].x * L[j][i].x + B[j][c].y * L[j][i].y);
        lx.y = lx.y - (-B[j][c].x * L[j][i].y + B[j][c].y * L[j][i].x);
      }
      help = (L[i][i].x * L[i][i].x + L[i][i].y * L[i][i].y);
      B[i][c].x = (lx.x * L[i][i].x - lx.y * L[i][i].y) / help;
      B[i][c].y = (lx.y * L[i][i].x + lx.x * L[i][i].y) / help;
    }
  }
}

}  // namespace crava
