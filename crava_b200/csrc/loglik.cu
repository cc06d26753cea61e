// loglik.cu -- Gaussian log marginal likelihood of the seismic spectra and
// its hand-written adjoint (gradients with respect to each angle's wavelet
// scale, noise variance and complex wavelet spectrum per kz).
//
// Model per inverted bin k (the per-bin algebra of the posterior solve,
// src/crava.cpp:1046-1135 of the reference): d = K m + e with
// m ~ CN(mu, S), e ~ CN(0, N), K = diag(w) A, so d ~ CN(K mu, M),
//   M_lm = w_l conj(w_m) B_lm + N_lm,   B = A S A^T,
//   N_lm = cc theta'_lm (e1_l conj(e1_m) + e2_l conj(e2_m))
//          + [l == m] wnc theta'_ll e3_l^2,   cc = (1 - wnc) |ec| / 2,
//   w_l(kz) = s_l D(kz) conj(W_l(kz)),  D(kz) = exp(2 pi i kz / nzp) - 1,
//   theta'_lm = theta_lm sqrt(v_l v_m / (theta_ll theta_mm)).
// The functional is
//   L = sum_k c_k (-log det M_k - r_k^H M_k^-1 r_k),  r = d - K mu,
// over the stored half spectrum with c_k = 2 for 0 < kx < nxp/2 (the bin
// stands for its conjugate partner too) and 1 on the kx = 0 and Nyquist
// planes; the constant -ntheta log(pi) per bin is left out.  Band-gated
// planes and bins whose M fails to factor do not enter.
//
// Adjoint (alpha = M^-1 r, G = alpha alpha^H - M^-1):
//   dL = tr(G dM) - 2 Re(alpha^H dr) = 2 Re sum_l u_l dw_l + (noise part),
//   u_l = sum_m G_ml conj(w_m) B_lm + conj(alpha_l) (A mu)_l,
//   dL/dRe w_l + i dL/dIm w_l = 2 conj(u_l),
//   dL/ds_l = 2 Re(w_l u_l) / s_l,
//   dL/dv_j = Re(sum_m G_mj N_jm) / v_j,
// and, through w(kz) = s D(kz) conj(W(kz)), w(nzp-kz) = s D(nzp-kz) W(kz),
//   dL/dW(kz) = s [D(kz) conj(g_w(kz)) + conj(D(nzp-kz)) g_w(nzp-kz)]
// (the second term for 0 < kz < nzp - kz).  The backward pass recomputes
// M and its factor per bin; nothing of the forward is stored.  FP64
// throughout, from the FP32 spectra.
#include <math.h>

#include <vector>

#include "context.cuh"
#include "solve_bin.cuh"

using namespace crava;

namespace {

constexpr int kThreads = 256;
using sb::tri;

__device__ __forceinline__ double2 dconj(double2 a) { return make_double2(a.x, -a.y); }

struct LLArgs {
  SolveConsts c;          // A, theta (already with the noise variances applied), wnc, var0
  const float2 *mu[3];
  const float2 *data[CRAVA_GPU_MAX_THETA];
  const float2 *cov[6];
  const float2 *err;
  const double2 *w;       // [nzp][nt] w_l(kz), scale included
  const float2 *e1, *e2;  // [nzp][nt]
  const float *e3;        // [nzp][nt]
  const int *inv;         // [nzp]
  double inv_s[CRAVA_GPU_MAX_THETA];  // 1 / s_l
  double inv_v[CRAVA_GPU_MAX_THETA];  // 1 / v_l
  int cnxp, nxp;
  long long plane;
  int bpp;                // blocks per kz plane
  double *part;           // [nzp][bpp][1 + 4 nt]
  unsigned long long *fail;
};

template <int NT>
__global__ void __launch_bounds__(kThreads) k_loglik(const __grid_constant__ LLArgs a) {
  constexpr int NV = 1 + 4 * NT;  // L, g_s[NT], g_v[NT], g_w[NT] (re, im)
  const int kz = blockIdx.y;
  double acc[NV];
#pragma unroll
  for (int t = 0; t < NV; ++t) acc[t] = 0.0;
  unsigned nfail = 0;
  if (a.inv[kz]) {
    double2 w[NT];
    float2 e1[NT], e2[NT];
    float e3[NT];
#pragma unroll
    for (int l = 0; l < NT; ++l) {
      w[l] = a.w[(long long)kz * NT + l];
      e1[l] = a.e1[(long long)kz * NT + l];
      e2[l] = a.e2[(long long)kz * NT + l];
      e3[l] = a.e3[(long long)kz * NT + l];
    }
    const SolveConsts &c = a.c;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < a.plane;
         i += (long long)a.bpp * blockDim.x) {
      const long long idx = (long long)kz * a.plane + i;
      const int kx = (int)(i % a.cnxp);
      const double ck = (kx == 0 || 2 * kx == a.nxp) ? 1.0 : 2.0;
      float2 c6[6];
#pragma unroll
      for (int t = 0; t < 6; ++t) c6[t] = a.cov[t][idx];
      const sb::Sym3d S = sb::prior_d(c6, c.var0);
      const float2 ec = a.err[idx];
      const double cc = 0.5 * (1.0 - (double)c.wnc) * fabs((double)ec.x);
      // (A mu)_l and r_l = d_l - w_l (A mu)_l
      double2 am[NT], r[NT];
      {
        double2 m3[3];
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          const float2 v = a.mu[q][idx];
          m3[q] = make_double2(v.x, v.y);
        }
#pragma unroll
        for (int l = 0; l < NT; ++l) {
          am[l] = make_double2(0.0, 0.0);
#pragma unroll
          for (int q = 0; q < 3; ++q)
            am[l] = dadd(am[l], make_double2(c.A[l][q] * m3[q].x, c.A[l][q] * m3[q].y));
          const float2 dl = a.data[l][idx];
          r[l] = dsub(make_double2(dl.x, dl.y), dmul(w[l], am[l]));
        }
      }
      // B = A S A^T (lower triangle) and M
      double B[NT * (NT + 1) / 2];
      double2 L[NT * (NT + 1) / 2];
#pragma unroll
      for (int l = 0; l < NT; ++l) {
        double as0 = 0, as1 = 0, as2 = 0;
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          as0 += (double)c.A[l][q] * sb::sget(S, q, 0);
          as1 += (double)c.A[l][q] * sb::sget(S, q, 1);
          as2 += (double)c.A[l][q] * sb::sget(S, q, 2);
        }
#pragma unroll
        for (int m = 0; m <= l; ++m) {
          const double b = as0 * c.A[m][0] + as1 * c.A[m][1] + as2 * c.A[m][2];
          B[tri(l, m)] = b;
          const double2 ww = dmulc(w[l], w[m]);
          const double2 n1 = dmulc(make_double2(e1[l].x, e1[l].y), make_double2(e1[m].x, e1[m].y));
          const double2 n2 = dmulc(make_double2(e2[l].x, e2[l].y), make_double2(e2[m].x, e2[m].y));
          const double f = cc * c.theta[l][m];
          double2 v = make_double2(ww.x * b + f * (n1.x + n2.x), ww.y * b + f * (n1.y + n2.y));
          if (l == m) {
            v.x += (double)c.wnc * c.theta[l][l] * (double)e3[l] * (double)e3[l];
            v.y = 0.0;
          }
          L[tri(l, m)] = v;
        }
      }
      double rd[NT];
      if (!sb::cholesky<NT, double2, double>(L, rd)) { ++nfail; continue; }
      // alpha = M^-1 r
      double2 al[NT];
#pragma unroll
      for (int i2 = 0; i2 < NT; ++i2) {
        double2 s = r[i2];
#pragma unroll
        for (int j = 0; j < i2; ++j) s = dsub(s, dmul(L[tri(i2, j)], al[j]));
        al[i2] = make_double2(s.x * rd[i2], s.y * rd[i2]);
      }
#pragma unroll
      for (int i2 = NT - 1; i2 >= 0; --i2) {
        double2 s = al[i2];
#pragma unroll
        for (int j = i2 + 1; j < NT; ++j) {
          const double2 lji = L[tri(j, i2)], x = al[j];  // conj(lji) x
          s.x -= lji.x * x.x + lji.y * x.y;
          s.y -= lji.x * x.y - lji.y * x.x;
        }
        al[i2] = make_double2(s.x * rd[i2], s.y * rd[i2]);
      }
      double logdet = 0.0, quad = 0.0;
#pragma unroll
      for (int l = 0; l < NT; ++l) {
        logdet += 2.0 * log(L[tri(l, l)].x);
        quad += r[l].x * al[l].x + r[l].y * al[l].y;  // Re(conj(r) alpha)
      }
      acc[0] += ck * (-logdet - quad);
      // Y = L^-1 (lower), M^-1 = Y^H Y, G = alpha alpha^H - M^-1 (lower)
      double2 Y[NT * (NT + 1) / 2];
#pragma unroll
      for (int j = 0; j < NT; ++j) {
        Y[tri(j, j)] = make_double2(rd[j], 0.0);
#pragma unroll
        for (int i2 = j + 1; i2 < NT; ++i2) {
          double2 s = make_double2(0.0, 0.0);
#pragma unroll
          for (int k = j; k < i2; ++k) s = dadd(s, dmul(L[tri(i2, k)], Y[tri(k, j)]));
          Y[tri(i2, j)] = make_double2(-s.x * rd[i2], -s.y * rd[i2]);
        }
      }
      double2 G[NT * (NT + 1) / 2];
#pragma unroll
      for (int l = 0; l < NT; ++l)
#pragma unroll
        for (int m = 0; m <= l; ++m) {
          double2 mi = make_double2(0.0, 0.0);
#pragma unroll
          for (int k = l; k < NT; ++k) mi = dadd(mi, dmulc(Y[tri(k, m)], Y[tri(k, l)]));  // conj(Y_kl) Y_km
          const double2 aa = dmulc(al[l], al[m]);
          G[tri(l, m)] = dsub(aa, mi);
        }
      // u_l and the accumulators
#pragma unroll
      for (int l = 0; l < NT; ++l) {
        double2 u = dmulc(am[l], al[l]);  // conj(alpha_l) (A mu)_l
        double gv = 0.0;
#pragma unroll
        for (int m = 0; m < NT; ++m) {
          const double2 Gml = m >= l ? G[tri(m, l)] : dconj(G[tri(l, m)]);
          const double b = m >= l ? B[tri(m, l)] : B[tri(l, m)];
          const double2 cw = make_double2(w[m].x * b, -w[m].y * b);  // conj(w_m) B_lm
          u = dadd(u, dmul(Gml, cw));
          // N_lm (row l = j of the noise gradient)
          double2 n;
          if (m == l) {
            n = make_double2(cc * c.theta[l][l] *
                                 ((double)e1[l].x * e1[l].x + (double)e1[l].y * e1[l].y +
                                  (double)e2[l].x * e2[l].x + (double)e2[l].y * e2[l].y) +
                             (double)c.wnc * c.theta[l][l] * (double)e3[l] * (double)e3[l],
                             0.0);
          } else {
            const double2 n1 = dmulc(make_double2(e1[l].x, e1[l].y), make_double2(e1[m].x, e1[m].y));
            const double2 n2 = dmulc(make_double2(e2[l].x, e2[l].y), make_double2(e2[m].x, e2[m].y));
            const double f = cc * c.theta[l][m];
            n = make_double2(f * (n1.x + n2.x), f * (n1.y + n2.y));
          }
          gv += Gml.x * n.x - Gml.y * n.y;  // Re(G_ml N_lm)
        }
        acc[1 + l] += ck * 2.0 * (w[l].x * u.x - w[l].y * u.y) * a.inv_s[l];
        acc[1 + NT + l] += ck * gv * a.inv_v[l];
        acc[1 + 2 * NT + 2 * l] += ck * 2.0 * u.x;
        acc[1 + 2 * NT + 2 * l + 1] += ck * (-2.0 * u.y);
      }
    }
  }
  // block reduction in a fixed order
  __shared__ double red[kThreads / 32][NV];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int t = 0; t < NV; ++t) {
    double v = acc[t];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) red[warp][t] = v;
  }
  unsigned fs = nfail;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) fs += __shfl_down_sync(0xffffffffu, fs, o);
  if (lane == 0 && fs) atomicAdd(a.fail, (unsigned long long)fs);
  __syncthreads();
  if (threadIdx.x < NV) {
    double v = 0.0;
    for (int wi = 0; wi < kThreads / 32; ++wi) v += red[wi][threadIdx.x];
    a.part[((long long)kz * a.bpp + blockIdx.x) * NV + threadIdx.x] = v;
  }
}

int launch_loglik(const LLArgs &a, int nt, int nzp, cudaStream_t s) {
  const dim3 grd((unsigned)a.bpp, (unsigned)nzp);
  switch (nt) {
#define CRAVA_LL_CASE(N) \
    case N: k_loglik<N><<<grd, kThreads, 0, s>>>(a); break;
    CRAVA_LL_CASE(1) CRAVA_LL_CASE(2) CRAVA_LL_CASE(3) CRAVA_LL_CASE(4)
    CRAVA_LL_CASE(5) CRAVA_LL_CASE(6) CRAVA_LL_CASE(7) CRAVA_LL_CASE(8)
#undef CRAVA_LL_CASE
    default: return CRAVA_GPU_ERR_ARG;
  }
  CRAVA_LAUNCH_CHECK();
  return CRAVA_GPU_OK;
}

// Unnormalised forward DFT of the context's wavelets (Wavelet::fft1DInPlace)
// in double, kz = 0 .. nzp/2: [cnzp][nt] (re, im).
std::vector<double> wavelet_spectrum(const crava_gpu_ctx *c) {
  const int nzp = c->p.nzp, nt = c->p.ntheta, cn = nzp / 2 + 1;
  std::vector<double> W((size_t)cn * nt * 2);
  for (int l = 0; l < nt; ++l)
    for (int k = 0; k < cn; ++k) {
      double re = 0, im = 0;
      for (int n = 0; n < nzp; ++n) {
        const long long m = ((long long)k * n) % nzp;
        const double ang = -2.0 * M_PI * (double)m / nzp;
        const double x = c->wavelet[(size_t)l * nzp + n];
        re += x * cos(ang);
        im += x * sin(ang);
      }
      W[((size_t)k * nt + l) * 2] = re;
      W[((size_t)k * nt + l) * 2 + 1] = im;
    }
  return W;
}

}  // namespace

extern "C" int crava_gpu_loglik_grad(crava_gpu_ctx *c, const crava_gpu_grids *gr,
                                     const double *wavelet_scale, const double *noise_var,
                                     const double *wavelet_spec, double *loglik, double *g_scale,
                                     double *g_noise, double *g_spec, long long *failed_bins) {
  int rc;
  if (!c || !loglik) return CRAVA_GPU_ERR_ARG;
  if ((rc = check_grids(c, gr))) return rc;
  const int nt = c->p.ntheta, nzp = c->p.nzp, cn = nzp / 2 + 1;
  std::vector<double> s(nt, 1.0), v(nt);
  for (int l = 0; l < nt; ++l) {
    v[l] = c->consts.theta[l][l];
    if (wavelet_scale) s[l] = wavelet_scale[l];
    if (noise_var) v[l] = noise_var[l];
    if (!(s[l] != 0.0) || !(v[l] > 0.0) || !(c->consts.theta[l][l] > 0.0)) return CRAVA_GPU_ERR_ARG;
  }
  std::vector<double> W = wavelet_spec ? std::vector<double>(wavelet_spec, wavelet_spec + (size_t)cn * nt * 2)
                                       : wavelet_spectrum(c);
  // w_l(kz) = s_l D(kz) conj(W_l(kz)), mirrored above nzp/2
  std::vector<double> D((size_t)nzp * 2), w((size_t)nzp * nt * 2);
  for (int k = 0; k < nzp; ++k) {
    const double ang = 2.0 * M_PI * (double)k / nzp;
    D[2 * k] = cos(ang) - 1.0;
    D[2 * k + 1] = sin(ang);
    for (int l = 0; l < nt; ++l) {
      const int kk = k < cn ? k : nzp - k;
      double wr = W[((size_t)kk * nt + l) * 2], wi = W[((size_t)kk * nt + l) * 2 + 1];
      if (k < cn) wi = -wi;  // conj(W(k)); above nzp/2 conj(W(nzp-k)) conjugated back
      const double dr = D[2 * k], di = D[2 * k + 1];
      w[((size_t)k * nt + l) * 2] = s[l] * (dr * wr - di * wi);
      w[((size_t)k * nt + l) * 2 + 1] = s[l] * (dr * wi + di * wr);
    }
  }
  DeviceGuard guard(c->device);
  LLArgs a{};
  a.c = c->consts;
  for (int l = 0; l < nt; ++l)
    for (int m = 0; m < nt; ++m)
      a.c.theta[l][m] = c->consts.theta[l][m] *
                        sqrt(v[l] * v[m] / (c->consts.theta[l][l] * c->consts.theta[m][m]));
  for (int q = 0; q < 3; ++q) a.mu[q] = reinterpret_cast<const float2 *>(gr->mu[q]);
  for (int l = 0; l < nt; ++l) a.data[l] = reinterpret_cast<const float2 *>(gr->data[l]);
  for (int t = 0; t < 6; ++t) a.cov[t] = reinterpret_cast<const float2 *>(gr->cov[t]);
  a.err = reinterpret_cast<const float2 *>(gr->err_corr);
  a.e1 = c->tables.e1; a.e2 = c->tables.e2; a.e3 = c->tables.e3; a.inv = c->tables.inv;
  for (int l = 0; l < nt; ++l) { a.inv_s[l] = 1.0 / s[l]; a.inv_v[l] = 1.0 / v[l]; }
  a.cnxp = c->g.cnxp; a.nxp = c->g.nxp;
  a.plane = (long long)c->g.cnxp * c->g.nyp;
  const long long per_plane_blocks = (a.plane + kThreads - 1) / kThreads;
  long long bpp = (4LL * 148 + nzp - 1) / nzp;
  if (bpp > per_plane_blocks) bpp = per_plane_blocks;
  if (bpp < 1) bpp = 1;
  a.bpp = (int)bpp;
  const int NV = 1 + 4 * nt;
  const size_t part_n = (size_t)nzp * a.bpp * NV;
  // the operator table, the partial sums and the failure count live in one
  // device buffer kept on the context (grown when a call needs more), the
  // partial sums come back into a pinned host buffer: no allocation, and no
  // device-wide synchronisation, after the first call
  const size_t w_bytes = (w.size() * sizeof(double) + 255) / 256 * 256;
  const size_t p_bytes = (part_n * sizeof(double) + 255) / 256 * 256;
  const size_t need = w_bytes + p_bytes + 256;
  const size_t host_need = p_bytes + 256;
  if (c->ll_bytes < need) {
    cudaFree(c->ll_buf);
    c->ll_buf = nullptr;
    c->ll_bytes = 0;
    if (cudaMalloc(&c->ll_buf, need) != cudaSuccess) return CRAVA_GPU_ERR_ALLOC;
    c->ll_bytes = need;
  }
  if (c->ll_host_bytes < host_need) {
    if (c->ll_host) cudaFreeHost(c->ll_host);
    c->ll_host = nullptr;
    c->ll_host_bytes = 0;
    if (cudaMallocHost(&c->ll_host, host_need) != cudaSuccess) return CRAVA_GPU_ERR_ALLOC;
    c->ll_host_bytes = host_need;
  }
  double2 *dw = reinterpret_cast<double2 *>(c->ll_buf);
  double *dpart = reinterpret_cast<double *>(c->ll_buf + w_bytes);
  unsigned long long *dfail = reinterpret_cast<unsigned long long *>(c->ll_buf + w_bytes + p_bytes);
  const double *part = reinterpret_cast<const double *>(c->ll_host);
  const unsigned long long *hfail_p = reinterpret_cast<const unsigned long long *>(c->ll_host + p_bytes);
  cudaError_t e = cudaMemcpyAsync(dw, w.data(), w.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(dfail, 0, sizeof(unsigned long long), c->stream);
  if (e != cudaSuccess) { set_last_error(e, "loglik upload", __FILE__, __LINE__); return CRAVA_GPU_ERR_CUDA; }
  a.w = dw; a.part = dpart; a.fail = dfail;
  // stage events around the kernel: crava_gpu_get_stats then reports its
  // device time as ms_solve and ms_total
  if ((rc = stage_event(c, 0)) || (rc = stage_event(c, 1))) return rc;
  if ((rc = launch_loglik(a, nt, nzp, c->stream))) return rc;
  if ((rc = stage_event(c, 2)) || (rc = stage_event(c, 3))) return rc;
  c->timed = true;
  e = cudaMemcpyAsync(c->ll_host, dpart, part_n * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(c->ll_host + p_bytes, dfail, sizeof(unsigned long long), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) { set_last_error(e, "loglik download", __FILE__, __LINE__); return CRAVA_GPU_ERR_CUDA; }
  const unsigned long long hfail = *hfail_p;
  // fixed-order reduction on the host
  double Lsum = 0.0;
  std::vector<double> gs(nt, 0.0), gv(nt, 0.0), gw((size_t)nzp * nt * 2, 0.0);
  for (int k = 0; k < nzp; ++k)
    for (int b = 0; b < a.bpp; ++b) {
      const double *p = &part[((size_t)k * a.bpp + b) * NV];
      Lsum += p[0];
      for (int l = 0; l < nt; ++l) {
        gs[l] += p[1 + l];
        gv[l] += p[1 + nt + l];
        gw[((size_t)k * nt + l) * 2] += p[1 + 2 * nt + 2 * l];
        gw[((size_t)k * nt + l) * 2 + 1] += p[1 + 2 * nt + 2 * l + 1];
      }
    }
  *loglik = Lsum;
  if (failed_bins) *failed_bins = (long long)hfail;
  if (g_scale) for (int l = 0; l < nt; ++l) g_scale[l] = gs[l];
  if (g_noise) for (int l = 0; l < nt; ++l) g_noise[l] = gv[l];
  if (g_spec) {
    for (int k = 0; k < cn; ++k)
      for (int l = 0; l < nt; ++l) {
        const double gr_ = gw[((size_t)k * nt + l) * 2], gi = gw[((size_t)k * nt + l) * 2 + 1];
        // s D(k) conj(g_w(k))
        double re = s[l] * (D[2 * k] * gr_ + D[2 * k + 1] * gi);
        double im = s[l] * (D[2 * k + 1] * gr_ - D[2 * k] * gi);
        const int km = nzp - k;
        if (k > 0 && km != k) {
          // s conj(D(nzp-k)) g_w(nzp-k)
          const double hr = gw[((size_t)km * nt + l) * 2], hi = gw[((size_t)km * nt + l) * 2 + 1];
          re += s[l] * (D[2 * km] * hr + D[2 * km + 1] * hi);
          im += s[l] * (D[2 * km] * hi - D[2 * km + 1] * hr);
        }
        g_spec[((size_t)k * nt + l) * 2] = re;
        g_spec[((size_t)k * nt + l) * 2 + 1] = im;
      }
  }
  return CRAVA_GPU_OK;
}
