// solve_ref.cu -- FP32 per-bin posterior solve in the reference's own float
// arithmetic and operation order.
//
// Compiled with -fmad=false (no multiply-add contraction) so that each float
// operation rounds once, as the reference's x86 build does.  With identical
// Fourier-domain inputs and per-kz tables the outputs equal those of the
// reference loop bit for bit.  Follows src/crava.cpp:1085-1151 with
// lib_matrProdCpx, lib_matrProdAdjointCpx, lib_matrAddMatCpx,
// lib_matrCholCpx (libs/lib/lib_matr.c:78-167), lib_matrAdjoint,
// lib_matrAXeqBMatCpx (:330-365), lib_matrSubtMatCpx, lib_matrProdMatVecCpx,
// lib_matrSubtVecCpx, lib_matrProdAdjointMatVecCpx, lib_matrAddVecCpx,
// getNextParameterCovariance (src/seismicparametersholder.cpp:355-427) and
// getNextErrorVariance (src/crava.cpp:1297-1334).
#include <math.h>

#include "lib_matr_ref.cuh"
#include "solve.cuh"

namespace crava {

namespace {

constexpr int kThreads = 128;

struct RefArgs {
  SolveConsts c;
  SolveGrids g;
  KzTables t;
  long long csize, plane;
  DevCounters *counters;
};

template <int NT>
__global__ void __launch_bounds__(kThreads) k_solve_ref(RefArgs a) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= a.csize) return;
  const int k = (int)(idx / a.plane);
  const SolveConsts &c = a.c;
  float2 mean[3], dat[NT], res[NT], S[3][3];
#pragma unroll
  for (int q = 0; q < 3; ++q) mean[q] = a.g.mu[q][idx];
#pragma unroll
  for (int l = 0; l < NT; ++l) { dat[l] = a.g.data[l][idx]; res[l] = dat[l]; }
  {
    const int ip[6] = {0, 1, 2, 0, 0, 1}, iq[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
    for (int t = 0; t < 6; ++t) {
      float2 cv = a.g.cov[t][idx];
      float v = (float)c.var0[t];
      float x = cv.x;
      if (c.var0[t] != 0) x = x / v;
      float aa = sqrtf(x * x);
      S[ip[t]][iq[t]] = make_float2(aa * v, 0.0f);
      if (ip[t] != iq[t]) S[iq[t]][ip[t]] = make_float2(aa * v, -0.0f);
    }
  }
  const float2 ec = a.g.err[idx];
  const float lam = sqrtf(ec.x * ec.x);
  bool fail = false;
  if (a.t.inv[k]) {
    float2 K[NT][3], KS[NT][3], KScc[3][NT], M[NT][NT], R[3][3], dm[NT], ans[3];
    float2 e1[NT], e2[NT];
    float e3[NT];
#pragma unroll
    for (int l = 0; l < NT; ++l) {
      float2 w = __ldg(a.t.wd + (long long)k * NT + l);
      e1[l] = __ldg(a.t.e1 + (long long)k * NT + l);
      e2[l] = __ldg(a.t.e2 + (long long)k * NT + l);
      e3[l] = __ldg(a.t.e3 + (long long)k * NT + l);
#pragma unroll
      for (int q = 0; q < 3; ++q) K[l][q] = make_float2(w.x * c.A[l][q], w.y * c.A[l][q]);
    }
    const double wnc = c.wnc;
#pragma unroll
    for (int l = 0; l < NT; ++l)
#pragma unroll
      for (int m = 0; m < NT; ++m) {
        double th = c.theta[l][m];
        float2 E;
        E.x = (float)(0.5 * (1.0 - wnc) * th * lam * (e1[l].x * e1[m].x + e1[l].y * e1[m].y));
        E.x += (float)(0.5 * (1.0 - wnc) * th * lam * (e2[l].x * e2[m].x + e2[l].y * e2[m].y));
        if (l == m) {
          E.x += (float)(wnc * th * e3[l] * e3[l]);
          E.y = 0.0f;
        } else {
          E.y = (float)(0.5 * (1.0 - wnc) * th * lam * (-e1[l].x * e1[m].y + e1[l].y * e1[m].x));
          E.y += (float)(0.5 * (1.0 - wnc) * th * lam * (-e2[l].x * e2[m].y + e2[l].y * e2[m].x));
        }
        M[l][m] = E;  // errVar, added below
      }
#pragma unroll
    for (int l = 0; l < NT; ++l)
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        float2 x = make_float2(0.0f, 0.0f);
#pragma unroll
        for (int r = 0; r < 3; ++r) {
          x.x += K[l][r].x * S[r][q].x - K[l][r].y * S[r][q].y;
          x.y += K[l][r].y * S[r][q].x + K[l][r].x * S[r][q].y;
        }
        KS[l][q] = x;
      }
#pragma unroll
    for (int l = 0; l < NT; ++l)
#pragma unroll
      for (int m = 0; m < NT; ++m) {
        float2 x = make_float2(0.0f, 0.0f);
#pragma unroll
        for (int r = 0; r < 3; ++r) {
          x.x += KS[l][r].x * K[m][r].x + KS[l][r].y * K[m][r].y;
          x.y += KS[l][r].y * K[m][r].x - KS[l][r].x * K[m][r].y;
        }
        // margVar = KS K^H, then margVar += errVar (lib_matrAddMatCpx: y += x)
        float2 e = M[l][m];
        x.x += e.x; x.y += e.y;
        M[l][m] = x;
      }
    if (chol_ref<NT>(M) == 0) {
#pragma unroll
      for (int l = 0; l < NT; ++l)
#pragma unroll
        for (int q = 0; q < 3; ++q) KScc[q][l] = make_float2(KS[l][q].x, -KS[l][q].y);
      axeqb_ref<NT, 3>(M, KS);
#pragma unroll
      for (int p = 0; p < 3; ++p)
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          float2 x = make_float2(0.0f, 0.0f);
#pragma unroll
          for (int l = 0; l < NT; ++l) {
            x.x += KScc[p][l].x * KS[l][q].x - KScc[p][l].y * KS[l][q].y;
            x.y += KScc[p][l].y * KS[l][q].x + KScc[p][l].x * KS[l][q].y;
          }
          R[p][q] = x;
        }
#pragma unroll
      for (int p = 0; p < 3; ++p)
#pragma unroll
        for (int q = 0; q < 3; ++q) { S[p][q].x -= R[p][q].x; S[p][q].y -= R[p][q].y; }
#pragma unroll
      for (int l = 0; l < NT; ++l) {
        float2 x = make_float2(0.0f, 0.0f);
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          x.x += K[l][q].x * mean[q].x - K[l][q].y * mean[q].y;
          x.y += K[l][q].y * mean[q].x + K[l][q].x * mean[q].y;
        }
        dm[l] = x;
      }
#pragma unroll
      for (int l = 0; l < NT; ++l) { dat[l].x -= dm[l].x; dat[l].y -= dm[l].y; }
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        float2 x = make_float2(0.0f, 0.0f);
#pragma unroll
        for (int l = 0; l < NT; ++l) {
          x.x += KS[l][q].x * dat[l].x + KS[l][q].y * dat[l].y;
          x.y += -KS[l][q].y * dat[l].x + KS[l][q].x * dat[l].y;
        }
        ans[q] = x;
      }
#pragma unroll
      for (int q = 0; q < 3; ++q) { mean[q].x += ans[q].x; mean[q].y += ans[q].y; }
#pragma unroll
      for (int l = 0; l < NT; ++l) {
        float2 x = make_float2(0.0f, 0.0f);
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          x.x += K[l][q].x * mean[q].x - K[l][q].y * mean[q].y;
          x.y += K[l][q].y * mean[q].x + K[l][q].x * mean[q].y;
        }
        dat[l] = x;
      }
#pragma unroll
      for (int l = 0; l < NT; ++l) { res[l].x -= dat[l].x; res[l].y -= dat[l].y; }
    } else {
      fail = true;
    }
  }
  bool nonfinite = false;
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    a.g.mu[q][idx] = mean[q];
    nonfinite |= !(isfinite(mean[q].x) && isfinite(mean[q].y));
  }
  const float2 o6[6] = {S[0][0], S[1][1], S[2][2], S[0][1], S[0][2], S[1][2]};
#pragma unroll
  for (int t = 0; t < 6; ++t) {
    a.g.cov[t][idx] = o6[t];
    nonfinite |= !(isfinite(o6[t].x) && isfinite(o6[t].y));
  }
#pragma unroll
  for (int l = 0; l < NT; ++l) {
    a.g.data[l][idx] = res[l];
    nonfinite |= !(isfinite(res[l].x) && isfinite(res[l].y));
  }
  if (a.counters) {
    unsigned m = __activemask();
    unsigned bf = __ballot_sync(m, fail), bn = __ballot_sync(m, nonfinite);
    if ((threadIdx.x & 31) == __ffs(m) - 1) {
      if (bf) atomicAdd(&a.counters->chol_fail, (unsigned long long)__popc(bf));
      if (bn) atomicAdd(&a.counters->nonfinite, (unsigned long long)__popc(bn));
    }
  }
}

}  // namespace

int posterior_solve_fp32ref(const SolveConsts &c, const KzTables &t,
                            const SolveGrids &g, long long csize, long long plane,
                            DevCounters *counters, cudaStream_t s) {
  RefArgs a;
  a.c = c; a.g = g; a.t = t; a.csize = csize; a.plane = plane; a.counters = counters;
  dim3 grd((unsigned)((csize + kThreads - 1) / kThreads));
  switch (c.nt) {
    case 1: k_solve_ref<1><<<grd, kThreads, 0, s>>>(a); break;
    case 2: k_solve_ref<2><<<grd, kThreads, 0, s>>>(a); break;
    case 3: k_solve_ref<3><<<grd, kThreads, 0, s>>>(a); break;
    case 4: k_solve_ref<4><<<grd, kThreads, 0, s>>>(a); break;
    case 5: k_solve_ref<5><<<grd, kThreads, 0, s>>>(a); break;
    case 6: k_solve_ref<6><<<grd, kThreads, 0, s>>>(a); break;
    case 7: k_solve_ref<7><<<grd, kThreads, 0, s>>>(a); break;
    case 8: k_solve_ref<8><<<grd, kThreads, 0, s>>>(a); break;
    default: return CRAVA_GPU_ERR_ARG;
  }
  CRAVA_LAUNCH_CHECK();
  return CRAVA_GPU_OK;
}

}  // namespace crava
