/*
 * crava_oracle.c -- plain-C restatement of the reference's Fourier-domain
 * AVO inversion hot path.  TEST INFRASTRUCTURE ONLY (see crava_oracle.h):
 * the product never links or calls it.
 *
 * Each function names the reference file:line it restates.  The FP32 solve
 * keeps the reference's float operation order (lib_matr.c) so that, built
 * with -ffp-contract=off, it reproduces the reference harness bit for bit
 * on identical Fourier-domain inputs.  The FFT is an independent
 * double-precision mixed-radix DFT rounded to float, so FFT outputs agree
 * with FFTW 2.1.2 (single precision) to float rounding, not bit for bit.
 */
#include "crava_oracle.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORC_TOL 1e-20 /* libs/lib/lib_matr.c:20 */
#define ORC_MAXT 16

typedef struct { float re, im; } cf;
typedef struct { double re, im; } cd;

/* ------------------------------------------------------------------ */
/* 1-D complex DFT, double precision, recursive mixed radix.           */
/* sign = -1 forward (FFTW_FORWARD), +1 backward; unnormalised.        */
/* ------------------------------------------------------------------ */
static int smallest_factor(int n) {
  for (int p = 2; p * p <= n; ++p)
    if (n % p == 0) return p;
  return n;
}

static void dft_rec(const cd *in, int istride, cd *out, int n, int sign,
                    cd *tmp) {
  if (n == 1) { out[0] = in[0]; return; }
  int p = smallest_factor(n), m = n / p;
  for (int r = 0; r < p; ++r)
    dft_rec(in + (long)r * istride, istride * p, out + (long)r * m, m, sign, tmp);
  /* combine: X[k + m q] = sum_r W_n^{r (k + m q)} sub_r[k] */
  for (int k = 0; k < m; ++k) {
    for (int q = 0; q < p; ++q) {
      int kk = k + m * q;
      double sr = 0.0, si = 0.0;
      for (int r = 0; r < p; ++r) {
        long e = ((long)r * kk) % n;
        double ang = sign * 2.0 * M_PI * (double)e / (double)n;
        double c = cos(ang), s = sin(ang);
        cd v = out[(long)r * m + k];
        sr += v.re * c - v.im * s;
        si += v.re * s + v.im * c;
      }
      tmp[kk].re = sr; tmp[kk].im = si;
    }
  }
  memcpy(out, tmp, sizeof(cd) * n);
}

static void dft1d(cd *x, int n, int sign) {
  cd *in = (cd *)malloc(sizeof(cd) * n), *tmp = (cd *)malloc(sizeof(cd) * n);
  memcpy(in, x, sizeof(cd) * n);
  dft_rec(in, 1, x, n, sign, tmp);
  free(in); free(tmp);
}

/* ------------------------------------------------------------------ */
/* 3-D in-place R2C / C2R with FFTGrid scaling.                         */
/* fftInPlace: src/fftgrid.cpp:1803-1829; invFFTInPlace: :1831-1862;    */
/* transform: rfftw3d_create_plan(nzp,nyp,nxp) + rfftwnd_one_*          */
/* (libs/fft/rfftw/rfftwnd.c:180,558,564): real-to-half-complex along   */
/* x, complex along y and z, forward sign -, unnormalised.              */
/* ------------------------------------------------------------------ */
static void scale_real(float *g, long rsize, float s) {
  for (long i = 0; i < rsize; ++i) g[i] *= s; /* multiplyByScalar :1992 */
}

int orc_fft_r2c(float *grid, int nxp, int nyp, int nzp, int type) {
  int cnxp = nxp / 2 + 1, rnxp = 2 * cnxp;
  long rsize = (long)rnxp * nyp * nzp;
  if (type != ORC_COVARIANCE)
    scale_real(grid, rsize, 1.0f / sqrtf((float)(nxp * nyp * nzp)));
  int nmax = nxp > nyp ? nxp : nyp; if (nzp > nmax) nmax = nzp;
  cd *line = (cd *)malloc(sizeof(cd) * nmax);
  cf *c = (cf *)grid;
  /* x: real -> half complex, per (y,z) row */
  for (long row = 0; row < (long)nyp * nzp; ++row) {
    float *r = grid + row * rnxp;
    for (int i = 0; i < nxp; ++i) { line[i].re = r[i]; line[i].im = 0.0; }
    dft1d(line, nxp, -1);
    cf *o = c + row * cnxp;
    for (int i = 0; i < cnxp; ++i) { o[i].re = (float)line[i].re; o[i].im = (float)line[i].im; }
  }
  /* y and z: complex */
  for (int k = 0; k < nzp; ++k)
    for (int i = 0; i < cnxp; ++i) {
      cf *b = c + (long)k * cnxp * nyp + i;
      for (int j = 0; j < nyp; ++j) { line[j].re = b[(long)j * cnxp].re; line[j].im = b[(long)j * cnxp].im; }
      dft1d(line, nyp, -1);
      for (int j = 0; j < nyp; ++j) { b[(long)j * cnxp].re = (float)line[j].re; b[(long)j * cnxp].im = (float)line[j].im; }
    }
  for (int j = 0; j < nyp; ++j)
    for (int i = 0; i < cnxp; ++i) {
      cf *b = c + (long)j * cnxp + i;
      long st = (long)cnxp * nyp;
      for (int k = 0; k < nzp; ++k) { line[k].re = b[k * st].re; line[k].im = b[k * st].im; }
      dft1d(line, nzp, -1);
      for (int k = 0; k < nzp; ++k) { b[k * st].re = (float)line[k].re; b[k * st].im = (float)line[k].im; }
    }
  free(line);
  return 0;
}

int orc_fft_c2r(float *grid, int nxp, int nyp, int nzp, int type) {
  int cnxp = nxp / 2 + 1, rnxp = 2 * cnxp;
  long rsize = (long)rnxp * nyp * nzp;
  int nmax = nxp > nyp ? nxp : nyp; if (nzp > nmax) nmax = nzp;
  cd *line = (cd *)malloc(sizeof(cd) * nmax);
  cf *c = (cf *)grid;
  for (int j = 0; j < nyp; ++j)
    for (int i = 0; i < cnxp; ++i) {
      cf *b = c + (long)j * cnxp + i;
      long st = (long)cnxp * nyp;
      for (int k = 0; k < nzp; ++k) { line[k].re = b[k * st].re; line[k].im = b[k * st].im; }
      dft1d(line, nzp, +1);
      for (int k = 0; k < nzp; ++k) { b[k * st].re = (float)line[k].re; b[k * st].im = (float)line[k].im; }
    }
  for (int k = 0; k < nzp; ++k)
    for (int i = 0; i < cnxp; ++i) {
      cf *b = c + (long)k * cnxp * nyp + i;
      for (int j = 0; j < nyp; ++j) { line[j].re = b[(long)j * cnxp].re; line[j].im = b[(long)j * cnxp].im; }
      dft1d(line, nyp, +1);
      for (int j = 0; j < nyp; ++j) { b[(long)j * cnxp].re = (float)line[j].re; b[(long)j * cnxp].im = (float)line[j].im; }
    }
  /* x: half complex -> real.  The imaginary parts of the DC and (even nxp)
   * Nyquist terms are ignored, as a real-output inverse transform does. */
  double *xr = (double *)malloc(sizeof(double) * nxp);
  for (long row = 0; row < (long)nyp * nzp; ++row) {
    cf *in = c + row * cnxp;
    for (int i = 0; i < nxp; ++i) { line[i].re = 0; line[i].im = 0; }
    line[0].re = in[0].re;
    for (int i = 1; i < cnxp; ++i) {
      if (2 * i == nxp) { line[i].re = in[i].re; continue; }
      line[i].re = in[i].re; line[i].im = in[i].im;
      line[nxp - i].re = in[i].re; line[nxp - i].im = -in[i].im;
    }
    dft1d(line, nxp, +1);
    for (int i = 0; i < nxp; ++i) xr[i] = line[i].re;
    float *r = grid + row * rnxp;
    for (int i = 0; i < nxp; ++i) r[i] = (float)xr[i];
    r[nxp] = 0.0f;
    if (rnxp > nxp + 1) r[nxp + 1] = 0.0f;
  }
  free(xr); free(line);
  float scale;
  if (type == ORC_COVARIANCE) scale = (float)(1.0 / ((double)nxp * nyp * nzp));
  else scale = (float)(1.0 / sqrt((float)(nxp * nyp * nzp)));
  scale_real(grid, rsize, scale);
  return 0;
}

/* ------------------------------------------------------------------ */
/* Wavelet tables per kz.                                               */
/* ------------------------------------------------------------------ */
/* Wavelet::findNorm on a real wavelet (src/wavelet.cpp:789-808). */
static float time_norm(const float *w, int n) {
  double s = 0.0;
  for (int i = 0; i < n; ++i) s += (double)(w[i] * w[i]);
  return (float)sqrt(s);
}

/* Wavelet1D::fft1DInPlace (src/wavelet.cpp:246-261): unnormalised real
 * forward transform, nzp/2+1 coefficients. */
static void real_spectrum(const float *w, int n, cf *out) {
  cd *line = (cd *)malloc(sizeof(cd) * n);
  for (int i = 0; i < n; ++i) { line[i].re = w[i]; line[i].im = 0.0; }
  dft1d(line, n, -1);
  for (int i = 0; i < n / 2 + 1; ++i) { out[i].re = (float)line[i].re; out[i].im = (float)line[i].im; }
  free(line);
}

/* Wavelet::getCAmp(k) (src/wavelet.cpp:308-324): Hermitian mirror. */
static cf get_camp(const cf *s, int nzp, int k) {
  int cnzp = nzp / 2 + 1;
  cf v;
  if (k < cnzp) { v.re = s[k].re; v.im = s[k].im; }
  else { v.re = s[nzp - k].re; v.im = -s[nzp - k].im; }
  return v;
}

/* Wavelet::getCAmp(k, scale) (src/wavelet.cpp:327-385): the spectrum of
 * the wavelet stretched by `scale`, linear interpolation between bins. */
static cf get_camp_scaled(const cf *s, int nzp, int k, float scale) {
  int cnzp = nzp / 2 + 1, refk = k < cnzp ? k : nzp - k;
  cf v;
  float omega = (float)refk / scale;
  if (omega >= cnzp) { v.re = 0.0f; v.im = 0.0f; }
  else {
    int omL = (int)floorf(omega), omU = (int)floorf(omega) + 1;
    if (omU >= cnzp) omU -= 1;
    float dOmega = omega - (float)omL;
    v.re = s[omL].re * (1.0f - dOmega) + s[omU].re * dOmega;
    if (k < cnzp) v.im = (s[omL].im * (1.0f - dOmega) + s[omU].im * dOmega);
    else v.im = (-s[omL].im * (1.0f - dOmega) - s[omU].im * dOmega);
  }
  v.re /= scale; v.im /= scale;
  return v;
}

/* Crava::fillInverseAbskWRobust (src/crava.cpp:1358-1384) for one angle. */
static float inverse_abs_robust(const cf *W, int nzp, int k, float norm) {
  cf value = get_camp(W, nzp, k), valueFine = get_camp_scaled(W, nzp, k, 0.999f);
  float modulus = value.re * value.re + value.im * value.im;
  float modulusFine = valueFine.re * valueFine.re + valueFine.im * valueFine.im;
  float maxMod = modulus > modulusFine ? modulus : modulusFine;
  /* sqrt of a float argument resolves to the float overload in C++ */
  if (maxMod > 0.0) return (float)(1.0 / (double)sqrtf(maxMod));
  return norm * nzp * nzp * 100.0f;
}

/* errorSmooth3 = central(backward(forward(w))) -- the three Wavelet1D
 * difference constructors of src/wavelet1D.cpp:420-479. */
static void smooth3(const float *w, int n, float *g) {
  float *e = (float *)malloc(sizeof(float) * n), *f = (float *)malloc(sizeof(float) * n);
  for (int i = 0; i < n; ++i) e[i] = (i == n - 1) ? w[0] - w[i] : w[i + 1] - w[i];
  for (int i = 0; i < n; ++i) f[i] = (i == 0) ? e[0] - e[n - 1] : e[i] - e[i - 1];
  for (int i = 0; i < n; ++i) {
    if (i == 0) g[i] = (float)(0.5 * (f[1] - f[n - 1]));
    else if (i == n - 1) g[i] = (float)(0.5 * (f[0] - f[i - 1]));
    else g[i] = (float)(0.5 * (f[i + 1] - f[i - 1]));
  }
  free(e); free(f);
}

/* Builds the per-kz vectors of crava.cpp:1042-1058 (constant thickness):
 * fillkW (:1336-1344), diff1Operator (src/wavelet1D.cpp:368-394),
 * lib_matrProdScalVecCpx, fillkWNorm (:1346-1355), errMult3 = 1, and the
 * band gate (:1044,1098). */
int orc_kz_tables(const crava_oracle_params *p, float *wd_, float *e1_,
                  float *e2_, float *e3, int *inv) {
  int nzp = p->nzp, nt = p->ntheta, cnzp = nzp / 2 + 1;
  if (nt < 1 || nt > ORC_MAXT) return 1;
  cf *wd = (cf *)wd_, *e1 = (cf *)e1_, *e2 = (cf *)e2_;
  cf *W = (cf *)malloc(sizeof(cf) * cnzp * nt), *G = (cf *)malloc(sizeof(cf) * cnzp * nt);
  cf *D = (cf *)malloc(sizeof(cf) * cnzp);
  float *g = (float *)malloc(sizeof(float) * nzp), *dop = (float *)calloc(nzp, sizeof(float));
  float wn[ORC_MAXT], gn[ORC_MAXT];
  for (int l = 0; l < nt; ++l) {
    const float *w = p->wavelet + (long)l * nzp;
    wn[l] = p->wavelet_norm ? p->wavelet_norm[l] : time_norm(w, nzp);
    real_spectrum(w, nzp, W + (long)l * cnzp);
    smooth3(w, nzp, g);
    gn[l] = time_norm(g, nzp);
    real_spectrum(g, nzp, G + (long)l * cnzp);
  }
  dop[0] = -1.0f; dop[nzp - 1] = 1.0f;
  real_spectrum(dop, nzp, D);
  cf *D3 = (cf *)malloc(sizeof(cf) * cnzp);
  {
    /* diff3Operator = central(backward(diff1Operator)), src/crava.cpp:938-940 */
    float *d2 = (float *)malloc(sizeof(float) * nzp), *d3 = (float *)malloc(sizeof(float) * nzp);
    for (int i = 0; i < nzp; ++i) d2[i] = (i == 0) ? dop[0] - dop[nzp - 1] : dop[i] - dop[i - 1];
    for (int i = 0; i < nzp; ++i) {
      if (i == 0) d3[i] = (float)(0.5 * (d2[1] - d2[nzp - 1]));
      else if (i == nzp - 1) d3[i] = (float)(0.5 * (d2[0] - d2[i - 1]));
      else d3[i] = (float)(0.5 * (d2[i + 1] - d2[i - 1]));
    }
    real_spectrum(d3, nzp, D3);
    free(d2); free(d3);
  }
  for (int k = 0; k < nzp; ++k) {
    int mk = k < nzp - k ? k : nzp - k;
    float realFrequency = (float)((p->nz * 1000.0f) / (p->lz * nzp) * mk);
    inv[k] = (realFrequency > p->low_cut * p->min_rel_thick) && (realFrequency < p->high_cut);
    cf kD = get_camp(D, nzp, k);
    if (p->thickness_mode == 1) {
      /* non-constant thickness, src/crava.cpp:1059-1083 */
      cf kD3 = get_camp(D3, nzp, k);
      for (int l = 0; l < nt; ++l) {
        long o = (long)k * nt + l;
        wd[o] = kD;
        e1[o].re = 1.0f / wn[l]; e1[o].im = 0.0f;
        float m2 = 1.0f / gn[l];
        e2[o].re = kD3.re * m2; e2[o].im = kD3.im * m2;
        e3[o] = inverse_abs_robust(W + (long)l * cnzp, nzp, k, wn[l]);
      }
      continue;
    }
    for (int l = 0; l < nt; ++l) {
      cf a = get_camp(W + (long)l * cnzp, nzp, k);
      cf kw; kw.re = a.re; kw.im = -a.im;
      cf r; r.re = kD.re * kw.re - kD.im * kw.im; r.im = kD.re * kw.im + kD.im * kw.re;
      wd[(long)k * nt + l] = r;
      e1[(long)k * nt + l].re = a.re / wn[l];
      e1[(long)k * nt + l].im = -(a.im / wn[l]);
      cf b = get_camp(G + (long)l * cnzp, nzp, k);
      e2[(long)k * nt + l].re = b.re / gn[l];
      e2[(long)k * nt + l].im = -(b.im / gn[l]);
      e3[(long)k * nt + l] = 1.0f;
    }
  }
  free(W); free(G); free(D); free(D3); free(g); free(dop);
  return 0;
}

/* ------------------------------------------------------------------ */
/* FP32 complex kernels, float operation order of libs/lib/lib_matr.c   */
/* ------------------------------------------------------------------ */
/* lib_matrCholCpx, libs/lib/lib_matr.c:78-167 */
static int chol_f(int n, cf m[][ORC_MAXT]) {
  cf lr; float help;
  float factor = m[0][0].re;
  if (factor <= 0) return 1;
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) { m[i][j].re = m[i][j].re / factor; m[i][j].im = m[i][j].im / factor; }
  for (int i = 0; i < n; ++i) {
    if ((double)m[i][i].re <= ORC_TOL) return 1;
    for (int j = 0; j < i; ++j) {
      lr.re = 0.0f; lr.im = 0.0f;
      for (int k = 0; k < j; ++k) {
        lr.re += (m[i][k].re * m[j][k].re) + (m[i][k].im * m[j][k].im);
        lr.im += -(m[i][k].re * m[j][k].im) + (m[i][k].im * m[j][k].re);
      }
      help = m[j][j].re * m[j][j].re + m[j][j].im * m[j][j].im;
      m[i][j].re = ((m[i][j].re - lr.re) * m[j][j].re + (m[i][j].im - lr.im) * m[j][j].im) / help;
      /* the reference reads the just-updated real part here (:130) */
      m[i][j].im = ((m[i][j].im - lr.im) * m[j][j].re - (m[i][j].re - lr.re) * m[j][j].im) / help;
    }
    lr.re = 0.0f;
    for (int k = 0; k < i; ++k) lr.re += (m[i][k].re * m[i][k].re) + (m[i][k].im * m[i][k].im);
    lr.re = m[i][i].re - lr.re;
    if ((double)lr.re <= ORC_TOL) return 1;
    m[i][i].re = (float)sqrt(lr.re);
    m[i][i].im = 0.0f;
  }
  for (int i = 0; i < n; ++i)
    for (int j = 0; j <= i; ++j) {
      m[i][j].re *= (float)sqrt(factor);
      m[i][j].im *= (float)sqrt(factor);
    }
  return 0;
}

/* lib_matrAXeqBMatCpx, libs/lib/lib_matr.c:330-365 (B is n x nc) */
static void axeqb_f(int n, cf L[][ORC_MAXT], cf B[][3], int nc) {
  cf lx; float help;
  for (int c = 0; c < nc; ++c) {
    for (int i = 0; i < n; ++i) {
      lx = B[i][c];
      for (int j = 0; j < i; ++j) {
        lx.re -= (B[j][c].re * L[i][j].re - B[j][c].im * L[i][j].im);
        lx.im -= (B[j][c].im * L[i][j].re + B[j][c].re * L[i][j].im);
      }
      help = (L[i][i].re * L[i][i].re + L[i][i].im * L[i][i].im);
      B[i][c].re = (lx.re * L[i][i].re + lx.im * L[i][i].im) / help;
      B[i][c].im = (lx.im * L[i][i].re - lx.re * L[i][i].im) / help;
    }
    for (int i = n - 1; i >= 0; --i) {
      lx = B[i][c];
      for (int j = n - 1; j > i; --j) {
        lx.re = lx.re - (B[j][c].re * L[j][i].re + B[j][c].im * L[j][i].im);
        lx.im = lx.im - (-B[j][c].re * L[j][i].im + B[j][c].im * L[j][i].re);
      }
      help = (L[i][i].re * L[i][i].re + L[i][i].im * L[i][i].im);
      B[i][c].re = (lx.re * L[i][i].re - lx.im * L[i][i].im) / help;
      B[i][c].im = (lx.im * L[i][i].re + lx.re * L[i][i].im) / help;
    }
  }
}

/* getNextParameterCovariance, src/seismicparametersholder.cpp:355-427 */
static void prior3_f(const double *v0, const cf c[6], cf S[3][3]) {
  static const int ip[6] = {0, 1, 2, 0, 0, 1}, iq[6] = {0, 1, 2, 1, 2, 2};
  for (int t = 0; t < 6; ++t) {
    float v = (float)v0[ip[t] * 3 + iq[t]];
    float x = c[t].re;
    if (v0[ip[t] * 3 + iq[t]] != 0) x = x / v;
    float a = sqrtf(x * x);
    S[ip[t]][iq[t]].re = a * v; S[ip[t]][iq[t]].im = 0.0f;
    if (ip[t] != iq[t]) { S[iq[t]][ip[t]].re = a * v; S[iq[t]][ip[t]].im = -0.0f; }
  }
}

/* ------------------------------------------------------------------ */
/* Per-bin posterior, FP32, restating crava.cpp:1042-1151 with          */
/* getNextErrorVariance (:1297-1334).                                   */
/* ------------------------------------------------------------------ */
int orc_posterior_fp32_t(const crava_oracle_params *p, const float *wd_,
                         const float *e1_, const float *e2_, const float *e3,
                         const int *inv, float *const *mu_, float *const *data_,
                         float *const *cov_, const float *err_corr,
                         long long *chol_fail) {
  int nxp = p->nxp, nyp = p->nyp, nzp = p->nzp, nt = p->ntheta;
  int cnxp = nxp / 2 + 1;
  if (nt < 1 || nt > ORC_MAXT) return 1;
  const cf *wd = (const cf *)wd_, *e1 = (const cf *)e1_, *e2 = (const cf *)e2_;
  cf *mu[3], *data[ORC_MAXT], *cov[6];
  for (int q = 0; q < 3; ++q) mu[q] = (cf *)mu_[q];
  for (int l = 0; l < nt; ++l) data[l] = (cf *)data_[l];
  for (int q = 0; q < 6; ++q) cov[q] = (cf *)cov_[q];
  const cf *ec = (const cf *)err_corr;
  long long fails = 0;
  double wnc = p->wnc;
  cf K[ORC_MAXT][3], KS[ORC_MAXT][3], KScc[3][ORC_MAXT], M[ORC_MAXT][ORC_MAXT], E[ORC_MAXT][ORC_MAXT];
  cf S[3][3], R[3][3], mean[3], ans[3], dat[ORC_MAXT], res[ORC_MAXT], dm[ORC_MAXT];
  memset(E, 0, sizeof E); memset(ans, 0, sizeof ans);
  for (int k = 0; k < nzp; ++k) {
    const cf *w = wd + (long)k * nt, *m1 = e1 + (long)k * nt, *m2 = e2 + (long)k * nt;
    const float *m3 = e3 + (long)k * nt;
    for (int l = 0; l < nt; ++l)
      for (int q = 0; q < 3; ++q) { K[l][q].re = w[l].re * p->A[l * 3 + q]; K[l][q].im = w[l].im * p->A[l * 3 + q]; }
    for (int j = 0; j < nyp; ++j)
      for (int i = 0; i < cnxp; ++i) {
        long idx = i + (long)cnxp * (j + (long)nyp * k);
        for (int q = 0; q < 3; ++q) mean[q] = mu[q][idx];
        for (int l = 0; l < nt; ++l) { dat[l] = data[l][idx]; res[l] = dat[l]; }
        cf c6[6];
        for (int q = 0; q < 6; ++q) c6[q] = cov[q][idx];
        prior3_f(p->var0, c6, S);
        cf t = ec[idx];
        float lam = sqrtf(t.re * t.re);
        if (inv[k]) {
          for (int l = 0; l < nt; ++l)
            for (int m = 0; m < nt; ++m) {
              double th = p->theta_cov[l * nt + m];
              E[l][m].re = (float)(0.5 * (1.0 - wnc) * th * lam * (m1[l].re * m1[m].re + m1[l].im * m1[m].im));
              E[l][m].re += (float)(0.5 * (1.0 - wnc) * th * lam * (m2[l].re * m2[m].re + m2[l].im * m2[m].im));
              if (l == m) {
                E[l][m].re += (float)(wnc * th * m3[l] * m3[l]);
                E[l][m].im = 0.0f;
              } else {
                E[l][m].im = (float)(0.5 * (1.0 - wnc) * th * lam * (-m1[l].re * m1[m].im + m1[l].im * m1[m].re));
                E[l][m].im += (float)(0.5 * (1.0 - wnc) * th * lam * (-m2[l].re * m2[m].im + m2[l].im * m2[m].re));
              }
            }
          /* KS = K S  (lib_matrProdCpx) */
          for (int l = 0; l < nt; ++l)
            for (int q = 0; q < 3; ++q) {
              cf x = {0.0f, 0.0f};
              for (int r = 0; r < 3; ++r) {
                x.re += K[l][r].re * S[r][q].re - K[l][r].im * S[r][q].im;
                x.im += K[l][r].im * S[r][q].re + K[l][r].re * S[r][q].im;
              }
              KS[l][q] = x;
            }
          /* M = KS K^H (lib_matrProdAdjointCpx) ; M += E */
          for (int l = 0; l < nt; ++l)
            for (int m = 0; m < nt; ++m) {
              cf x = {0.0f, 0.0f};
              for (int r = 0; r < 3; ++r) {
                x.re += KS[l][r].re * K[m][r].re + KS[l][r].im * K[m][r].im;
                x.im += KS[l][r].im * K[m][r].re - KS[l][r].re * K[m][r].im;
              }
              M[l][m] = x;
            }
          for (int l = 0; l < nt; ++l)
            for (int m = 0; m < nt; ++m) { M[l][m].re += E[l][m].re; M[l][m].im += E[l][m].im; }
          int flag = chol_f(nt, M);
          if (flag == 0) {
            for (int l = 0; l < nt; ++l)
              for (int q = 0; q < 3; ++q) { KScc[q][l].re = KS[l][q].re; KScc[q][l].im = -KS[l][q].im; }
            axeqb_f(nt, M, KS, 3);
            for (int a = 0; a < 3; ++a)
              for (int b = 0; b < 3; ++b) {
                cf x = {0.0f, 0.0f};
                for (int l = 0; l < nt; ++l) {
                  x.re += KScc[a][l].re * KS[l][b].re - KScc[a][l].im * KS[l][b].im;
                  x.im += KScc[a][l].im * KS[l][b].re + KScc[a][l].re * KS[l][b].im;
                }
                R[a][b] = x;
              }
            for (int a = 0; a < 3; ++a)
              for (int b = 0; b < 3; ++b) { S[a][b].re -= R[a][b].re; S[a][b].im -= R[a][b].im; }
            for (int l = 0; l < nt; ++l) {
              cf x = {0.0f, 0.0f};
              for (int q = 0; q < 3; ++q) {
                x.re += K[l][q].re * mean[q].re - K[l][q].im * mean[q].im;
                x.im += K[l][q].im * mean[q].re + K[l][q].re * mean[q].im;
              }
              dm[l] = x;
            }
            for (int l = 0; l < nt; ++l) { dat[l].re -= dm[l].re; dat[l].im -= dm[l].im; }
            for (int q = 0; q < 3; ++q) {
              cf x = {0.0f, 0.0f};
              for (int l = 0; l < nt; ++l) {
                x.re += KS[l][q].re * dat[l].re + KS[l][q].im * dat[l].im;
                x.im += -KS[l][q].im * dat[l].re + KS[l][q].re * dat[l].im;
              }
              ans[q] = x;
            }
            for (int q = 0; q < 3; ++q) { mean[q].re += ans[q].re; mean[q].im += ans[q].im; }
            for (int l = 0; l < nt; ++l) {
              cf x = {0.0f, 0.0f};
              for (int q = 0; q < 3; ++q) {
                x.re += K[l][q].re * mean[q].re - K[l][q].im * mean[q].im;
                x.im += K[l][q].im * mean[q].re + K[l][q].re * mean[q].im;
              }
              dat[l] = x;
            }
            for (int l = 0; l < nt; ++l) { res[l].re -= dat[l].re; res[l].im -= dat[l].im; }
          } else {
            ++fails;
          }
        }
        for (int q = 0; q < 3; ++q) mu[q][idx] = mean[q];
        cov[0][idx] = S[0][0]; cov[1][idx] = S[1][1]; cov[2][idx] = S[2][2];
        cov[3][idx] = S[0][1]; cov[4][idx] = S[0][2]; cov[5][idx] = S[1][2];
        for (int l = 0; l < nt; ++l) data[l][idx] = res[l];
      }
  }
  if (chol_fail) *chol_fail = fails;
  return 0;
}

int orc_posterior_fp32(const crava_oracle_params *p, float *const *mu,
                       float *const *data, float *const *cov,
                       const float *err_corr, long long *chol_fail) {
  int nzp = p->nzp, nt = p->ntheta;
  if (nt < 1 || nt > ORC_MAXT) return 1;
  float *wd = (float *)malloc(sizeof(cf) * nzp * nt), *e1 = (float *)malloc(sizeof(cf) * nzp * nt);
  float *e2 = (float *)malloc(sizeof(cf) * nzp * nt);
  float *e3 = (float *)malloc(sizeof(float) * nzp * nt);
  int *inv = (int *)malloc(sizeof(int) * nzp);
  orc_kz_tables(p, wd, e1, e2, e3, inv);
  int rc = orc_posterior_fp32_t(p, wd, e1, e2, e3, inv, mu, data, cov, err_corr, chol_fail);
  free(wd); free(e1); free(e2); free(e3); free(inv);
  return rc;
}

/* ------------------------------------------------------------------ */
/* FP64 twin: the same algorithm (prior |Re| rule, M00 pre-scaled        */
/* Cholesky with the TOL test, substitutions, Schur update), carried in  */
/* double from the float spectra.                                        */
/* ------------------------------------------------------------------ */
static int chol_d(int n, cd m[][ORC_MAXT]) {
  double factor = m[0][0].re;
  if (factor <= 0) return 1;
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) { m[i][j].re /= factor; m[i][j].im /= factor; }
  for (int i = 0; i < n; ++i) {
    if (m[i][i].re <= ORC_TOL) return 1;
    for (int j = 0; j < i; ++j) {
      double lre = 0, lim = 0;
      for (int k = 0; k < j; ++k) {
        lre += m[i][k].re * m[j][k].re + m[i][k].im * m[j][k].im;
        lim += -m[i][k].re * m[j][k].im + m[i][k].im * m[j][k].re;
      }
      double h = m[j][j].re * m[j][j].re + m[j][j].im * m[j][j].im;
      double ar = m[i][j].re - lre, ai = m[i][j].im - lim;
      m[i][j].re = (ar * m[j][j].re + ai * m[j][j].im) / h;
      m[i][j].im = (ai * m[j][j].re - ar * m[j][j].im) / h;
    }
    double d = 0;
    for (int k = 0; k < i; ++k) d += m[i][k].re * m[i][k].re + m[i][k].im * m[i][k].im;
    d = m[i][i].re - d;
    if (d <= ORC_TOL) return 1;
    m[i][i].re = sqrt(d); m[i][i].im = 0.0;
  }
  double sf = sqrt(factor);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j <= i; ++j) { m[i][j].re *= sf; m[i][j].im *= sf; }
  return 0;
}

static void axeqb_d(int n, cd L[][ORC_MAXT], cd B[][3], int nc) {
  for (int c = 0; c < nc; ++c) {
    for (int i = 0; i < n; ++i) {
      double xr = B[i][c].re, xi = B[i][c].im;
      for (int j = 0; j < i; ++j) {
        xr -= B[j][c].re * L[i][j].re - B[j][c].im * L[i][j].im;
        xi -= B[j][c].im * L[i][j].re + B[j][c].re * L[i][j].im;
      }
      double h = L[i][i].re * L[i][i].re + L[i][i].im * L[i][i].im;
      B[i][c].re = (xr * L[i][i].re + xi * L[i][i].im) / h;
      B[i][c].im = (xi * L[i][i].re - xr * L[i][i].im) / h;
    }
    for (int i = n - 1; i >= 0; --i) {
      double xr = B[i][c].re, xi = B[i][c].im;
      for (int j = n - 1; j > i; --j) {
        xr -= B[j][c].re * L[j][i].re + B[j][c].im * L[j][i].im;
        xi -= -B[j][c].re * L[j][i].im + B[j][c].im * L[j][i].re;
      }
      double h = L[i][i].re * L[i][i].re + L[i][i].im * L[i][i].im;
      B[i][c].re = (xr * L[i][i].re - xi * L[i][i].im) / h;
      B[i][c].im = (xi * L[i][i].re + xr * L[i][i].im) / h;
    }
  }
}

int orc_posterior_fp64(const crava_oracle_params *p, const float *const *mu_,
                       const float *const *data_, const float *const *cov_,
                       const float *err_corr, double *const *mu_out,
                       double *const *cov_out, double *const *res_out,
                       long long *chol_fail) {
  int nxp = p->nxp, nyp = p->nyp, nzp = p->nzp, nt = p->ntheta;
  int cnxp = nxp / 2 + 1;
  if (nt < 1 || nt > ORC_MAXT) return 1;
  cf *wd = (cf *)malloc(sizeof(cf) * nzp * nt), *e1 = (cf *)malloc(sizeof(cf) * nzp * nt);
  cf *e2 = (cf *)malloc(sizeof(cf) * nzp * nt);
  float *e3 = (float *)malloc(sizeof(float) * nzp * nt);
  int *inv = (int *)malloc(sizeof(int) * nzp);
  orc_kz_tables(p, (float *)wd, (float *)e1, (float *)e2, e3, inv);
  static const int ip[6] = {0, 1, 2, 0, 0, 1}, iq[6] = {0, 1, 2, 1, 2, 2};
  long long fails = 0;
  double wnc = p->wnc;
  cd K[ORC_MAXT][3], KS[ORC_MAXT][3], KSo[ORC_MAXT][3], M[ORC_MAXT][ORC_MAXT];
  cd S[3][3], mean[3], dat[ORC_MAXT], res[ORC_MAXT];
  for (int k = 0; k < nzp; ++k) {
    const cf *w = wd + (long)k * nt, *m1 = e1 + (long)k * nt, *m2 = e2 + (long)k * nt;
    const float *m3 = e3 + (long)k * nt;
    for (int l = 0; l < nt; ++l)
      for (int q = 0; q < 3; ++q) { K[l][q].re = (double)w[l].re * p->A[l * 3 + q]; K[l][q].im = (double)w[l].im * p->A[l * 3 + q]; }
    for (int j = 0; j < nyp; ++j)
      for (int i = 0; i < cnxp; ++i) {
        long idx = i + (long)cnxp * (j + (long)nyp * k);
        for (int q = 0; q < 3; ++q) { const cf *g = (const cf *)mu_[q]; mean[q].re = g[idx].re; mean[q].im = g[idx].im; }
        for (int l = 0; l < nt; ++l) { const cf *g = (const cf *)data_[l]; dat[l].re = g[idx].re; dat[l].im = g[idx].im; res[l] = dat[l]; }
        for (int t = 0; t < 6; ++t) {
          const cf *g = (const cf *)cov_[t];
          double v = p->var0[ip[t] * 3 + iq[t]], x = g[idx].re;
          double a = (v != 0) ? fabs(x / v) * v : fabs(x);
          S[ip[t]][iq[t]].re = a; S[ip[t]][iq[t]].im = 0;
          S[iq[t]][ip[t]].re = a; S[iq[t]][ip[t]].im = 0;
        }
        double lam = fabs((double)((const cf *)err_corr)[idx].re);
        if (inv[k]) {
          for (int l = 0; l < nt; ++l)
            for (int m = 0; m < nt; ++m) {
              double th = p->theta_cov[l * nt + m], c = 0.5 * (1.0 - wnc) * th * lam;
              double er = c * ((double)m1[l].re * m1[m].re + (double)m1[l].im * m1[m].im)
                        + c * ((double)m2[l].re * m2[m].re + (double)m2[l].im * m2[m].im);
              double ei = 0.0;
              if (l == m) er += wnc * th * (double)m3[l] * m3[l];
              else ei = c * (-(double)m1[l].re * m1[m].im + (double)m1[l].im * m1[m].re)
                      + c * (-(double)m2[l].re * m2[m].im + (double)m2[l].im * m2[m].re);
              M[l][m].re = er; M[l][m].im = ei;
            }
          for (int l = 0; l < nt; ++l)
            for (int q = 0; q < 3; ++q) {
              double xr = 0, xi = 0;
              for (int r = 0; r < 3; ++r) {
                xr += K[l][r].re * S[r][q].re - K[l][r].im * S[r][q].im;
                xi += K[l][r].im * S[r][q].re + K[l][r].re * S[r][q].im;
              }
              KS[l][q].re = xr; KS[l][q].im = xi; KSo[l][q] = KS[l][q];
            }
          for (int l = 0; l < nt; ++l)
            for (int m = 0; m < nt; ++m) {
              double xr = 0, xi = 0;
              for (int r = 0; r < 3; ++r) {
                xr += KS[l][r].re * K[m][r].re + KS[l][r].im * K[m][r].im;
                xi += KS[l][r].im * K[m][r].re - KS[l][r].re * K[m][r].im;
              }
              M[l][m].re += xr; M[l][m].im += xi;
            }
          if (chol_d(nt, M) == 0) {
            axeqb_d(nt, M, KS, 3);
            for (int a = 0; a < 3; ++a)
              for (int b = 0; b < 3; ++b) {
                double xr = 0, xi = 0;
                for (int l = 0; l < nt; ++l) {
                  xr += KSo[l][a].re * KS[l][b].re + KSo[l][a].im * KS[l][b].im;
                  xi += KSo[l][a].re * KS[l][b].im - KSo[l][a].im * KS[l][b].re;
                }
                S[a][b].re -= xr; S[a][b].im -= xi;
              }
            cd dm[ORC_MAXT], ans[3];
            for (int l = 0; l < nt; ++l) {
              double xr = 0, xi = 0;
              for (int q = 0; q < 3; ++q) {
                xr += K[l][q].re * mean[q].re - K[l][q].im * mean[q].im;
                xi += K[l][q].im * mean[q].re + K[l][q].re * mean[q].im;
              }
              dm[l].re = dat[l].re - xr; dm[l].im = dat[l].im - xi;
            }
            for (int q = 0; q < 3; ++q) {
              double xr = 0, xi = 0;
              for (int l = 0; l < nt; ++l) {
                xr += KS[l][q].re * dm[l].re + KS[l][q].im * dm[l].im;
                xi += -KS[l][q].im * dm[l].re + KS[l][q].re * dm[l].im;
              }
              ans[q].re = xr; ans[q].im = xi;
            }
            for (int q = 0; q < 3; ++q) { mean[q].re += ans[q].re; mean[q].im += ans[q].im; }
            for (int l = 0; l < nt; ++l) {
              double xr = 0, xi = 0;
              for (int q = 0; q < 3; ++q) {
                xr += K[l][q].re * mean[q].re - K[l][q].im * mean[q].im;
                xi += K[l][q].im * mean[q].re + K[l][q].re * mean[q].im;
              }
              res[l].re -= xr; res[l].im -= xi;
            }
          } else {
            ++fails;
          }
        }
        for (int q = 0; q < 3; ++q) { mu_out[q][2 * idx] = mean[q].re; mu_out[q][2 * idx + 1] = mean[q].im; }
        for (int t = 0; t < 6; ++t) { cov_out[t][2 * idx] = S[ip[t]][iq[t]].re; cov_out[t][2 * idx + 1] = S[ip[t]][iq[t]].im; }
        for (int l = 0; l < nt; ++l) { res_out[l][2 * idx] = res[l].re; res_out[l][2 * idx + 1] = res[l].im; }
      }
  }
  if (chol_fail) *chol_fail = fails;
  free(wd); free(e1); free(e2); free(e3); free(inv);
  return 0;
}

/* ------------------------------------------------------------------ */
/* The timed unit: forward FFT of 3 means (PARAMETER), ntheta stacks     */
/* (DATA), 6 prior covariances and the noise correlation (COVARIANCE);   */
/* the solve; inverse FFT of 3 posterior means, ntheta residuals and 6   */
/* posterior covariances (crava.cpp:175-190, 1003, 1012, 1181-1206, 218).*/
/* ------------------------------------------------------------------ */
int orc_unit_fp32(const crava_oracle_params *p, float *const *mu,
                  float *const *data, float *const *cov, float *err_corr,
                  long long *chol_fail) {
  int nx = p->nxp, ny = p->nyp, nz = p->nzp;
  for (int q = 0; q < 3; ++q) orc_fft_r2c(mu[q], nx, ny, nz, ORC_PARAMETER);
  for (int l = 0; l < p->ntheta; ++l) orc_fft_r2c(data[l], nx, ny, nz, ORC_DATA);
  for (int q = 0; q < 6; ++q) orc_fft_r2c(cov[q], nx, ny, nz, ORC_COVARIANCE);
  orc_fft_r2c(err_corr, nx, ny, nz, ORC_COVARIANCE);
  int rc = orc_posterior_fp32(p, mu, data, cov, err_corr, chol_fail);
  for (int q = 0; q < 3; ++q) orc_fft_c2r(mu[q], nx, ny, nz, ORC_PARAMETER);
  for (int l = 0; l < p->ntheta; ++l) orc_fft_c2r(data[l], nx, ny, nz, ORC_DATA);
  for (int q = 0; q < 6; ++q) orc_fft_c2r(cov[q], nx, ny, nz, ORC_COVARIANCE);
  return rc;
}

/* ------------------------------------------------------------------ */
/* RNG: LCG x <- 69069 x + 1 (mod 2^32), u = x / 2^32, with the          */
/* Marsaglia-Bray normal generator (libs/lib/random.cpp:38-119,          */
/* constants libs/lib/random.h:12-15).                                   */
/* ------------------------------------------------------------------ */
typedef struct { uint32_t s; } lcg_t;
static double lcg_u(lcg_t *g) {
  g->s = 69069u * g->s + 1u;
  return (double)g->s * (1.0 / 4294967296.0);
}
static double mb_g(double x) {
  const double a = 17.49731196, b = 2.36785163, c = 2.15787544;
  double ax = fabs(x), r = a * exp(-x * x / 2.0);
  if (ax < 1.0) r -= 2.0 * b * (3.0 - x * x) + c * (1.5 - ax);
  else if (ax < 1.5) r -= b * (3.0 - ax) * (3.0 - ax) + c * (1.5 - ax);
  else r -= b * (3.0 - ax) * (3.0 - ax);
  return r;
}
static double lcg_norm(lcg_t *g) {
  double u = lcg_u(g), x;
  if (u < 0.8638) {
    double u1 = lcg_u(g), u2 = lcg_u(g), u3 = lcg_u(g);
    x = 2.0 * (u1 + u2 + u3) - 3.0;
  } else if (u < 0.9745) {
    double u1 = lcg_u(g), u2 = lcg_u(g);
    x = 1.5 * (u1 + u2 - 1.0);
  } else if (u < 0.9973002039) {
    double u1, u2;
    do { u1 = lcg_u(g); u2 = lcg_u(g); x = 6.0 * u1 - 3.0; } while (0.358 * u2 > mb_g(x));
  } else {
    double s, t;
    do {
      double v1, v2, w;
      do {
        double u1 = lcg_u(g), u2 = lcg_u(g);
        v1 = 2.0 * u1 - 1.0; v2 = 2.0 * u2 - 1.0; w = v1 * v1 + v2 * v2;
      } while (w >= 1.0);
      double c = sqrt((9.0 - 2.0 * log(w)) / w);
      s = c * v1; t = c * v2;
    } while (fabs(s) <= 3.0 && fabs(t) <= 3.0);
    x = fabs(s) > 3.0 ? s : t;
  }
  return x;
}

unsigned int orc_rng_fill_normal(unsigned int seed, double *out, long long n) {
  lcg_t g = {seed};
  for (long long i = 0; i < n; ++i) out[i] = lcg_norm(&g);
  return g.s;
}

/* FFTGrid::fillInComplexNoise, src/fftgrid.cpp:1213-1263 (including the
 * reference's parity test on the linear index for the last x plane). */
unsigned int orc_noise_fill(float *grid, int nxp, int nyp, int nzp,
                            unsigned int seed) {
  lcg_t g = {seed};
  int cnxp = nxp / 2 + 1;
  long csize = (long)cnxp * nyp * nzp;
  cf *c = (cf *)grid;
  float sd = (float)(1 / sqrt(2.0));
  for (long i = 0; i < csize; ++i) {
    if (((i % cnxp) == 0) || (((i % cnxp) == cnxp - 1) && ((i % 2) == 1))) {
      long xs = i % cnxp, jk = (i - xs) / cnxp;
      long jj = jk % nyp, kk = jk / nyp;
      long jc = jj == 0 ? 0 : nyp - jj, kc = kk == 0 ? 0 : nzp - kk;
      long jkc = jc + kc * nyp;
      if (jkc == jk) { c[i].re = (float)lcg_norm(&g); c[i].im = 0; }
      else if (jkc > jk) { c[i].re = (float)(sd * lcg_norm(&g)); c[i].im = (float)(sd * lcg_norm(&g)); }
      else { long ci = jkc * cnxp + xs; c[i].re = c[ci].re; c[i].im = -c[ci].im; }
    } else {
      c[i].re = (float)(sd * lcg_norm(&g));
      c[i].im = (float)(sd * lcg_norm(&g));
    }
  }
  return g.s;
}

/* Crava::simulate per-bin body, src/crava.cpp:1482-1521: rebuild the
 * Hermitian 3x3 from 6 posterior spectra, Cholesky, seed <- L seed
 * (lib_matrProdCholVec, lib_matr.c:453-470); zero on failure. */
int orc_sim_filter(int nxp, int nyp, int nzp, const float *const *cov_,
                   float *const *seed_, long long *chol_fail) {
  long csize = (long)(nxp / 2 + 1) * nyp * nzp;
  const cf *cv[6]; cf *sd[3];
  for (int t = 0; t < 6; ++t) cv[t] = (const cf *)cov_[t];
  for (int q = 0; q < 3; ++q) sd[q] = (cf *)seed_[q];
  long long fails = 0;
  cf P[ORC_MAXT][ORC_MAXT];
  for (long i = 0; i < csize; ++i) {
    P[0][0] = cv[0][i]; P[1][1] = cv[1][i]; P[2][2] = cv[2][i];
    P[0][1] = cv[3][i]; P[0][2] = cv[4][i]; P[1][2] = cv[5][i];
    P[1][0].re = P[0][1].re; P[1][0].im = -P[0][1].im;
    P[2][0].re = P[0][2].re; P[2][0].im = -P[0][2].im;
    P[2][1].re = P[1][2].re; P[2][1].im = -P[1][2].im;
    cf z[3] = {sd[0][i], sd[1][i], sd[2][i]}, o[3];
    if (chol_f(3, P) == 0) {
      for (int a = 0; a < 3; ++a) {
        o[a].re = 0.0f; o[a].im = 0.0f;
        for (int b = 0; b < a + 1; ++b) {
          o[a].re += P[a][b].re * z[b].re - P[a][b].im * z[b].im;
          o[a].im += P[a][b].re * z[b].im + P[a][b].im * z[b].re;
        }
      }
    } else {
      ++fails;
      for (int a = 0; a < 3; ++a) { o[a].re = 0.0f; o[a].im = 0.0f; }
    }
    for (int q = 0; q < 3; ++q) sd[q][i] = o[q];
  }
  if (chol_fail) *chol_fail = fails;
  return 0;
}

/* Same filter carried in double (for the GPU filter's tolerance check). */
int orc_sim_filter_fp64(int nxp, int nyp, int nzp, const float *const *cov_,
                        float *const *seed_, long long *chol_fail) {
  long csize = (long)(nxp / 2 + 1) * nyp * nzp;
  const cf *cv[6]; cf *sd[3];
  for (int t = 0; t < 6; ++t) cv[t] = (const cf *)cov_[t];
  for (int q = 0; q < 3; ++q) sd[q] = (cf *)seed_[q];
  long long fails = 0;
  cd P[ORC_MAXT][ORC_MAXT];
  for (long i = 0; i < csize; ++i) {
    const cf *src[6] = {cv[0] + i, cv[1] + i, cv[2] + i, cv[3] + i, cv[4] + i, cv[5] + i};
    P[0][0].re = src[0]->re; P[0][0].im = src[0]->im;
    P[1][1].re = src[1]->re; P[1][1].im = src[1]->im;
    P[2][2].re = src[2]->re; P[2][2].im = src[2]->im;
    P[0][1].re = src[3]->re; P[0][1].im = src[3]->im;
    P[0][2].re = src[4]->re; P[0][2].im = src[4]->im;
    P[1][2].re = src[5]->re; P[1][2].im = src[5]->im;
    P[1][0].re = P[0][1].re; P[1][0].im = -P[0][1].im;
    P[2][0].re = P[0][2].re; P[2][0].im = -P[0][2].im;
    P[2][1].re = P[1][2].re; P[2][1].im = -P[1][2].im;
    cd z[3];
    for (int q = 0; q < 3; ++q) { z[q].re = sd[q][i].re; z[q].im = sd[q][i].im; }
    if (chol_d(3, P) == 0) {
      for (int a = 0; a < 3; ++a) {
        double xr = 0, xi = 0;
        for (int b = 0; b <= a; ++b) {
          xr += P[a][b].re * z[b].re - P[a][b].im * z[b].im;
          xi += P[a][b].re * z[b].im + P[a][b].im * z[b].re;
        }
        sd[a][i].re = (float)xr; sd[a][i].im = (float)xi;
      }
    } else {
      ++fails;
      for (int a = 0; a < 3; ++a) { sd[a][i].re = 0.0f; sd[a][i].im = 0.0f; }
    }
  }
  if (chol_fail) *chol_fail = fails;
  return 0;
}

/* ------------------------------------------------------------------ */
/* Synthetic seismic: Crava::computeSyntSeismic (src/crava.cpp:1666-1719)
 * with computeSeismicImpedance (:1632-1663), constant thickness: per
 * angle, the impedance combination on every real cell; per trace
 * x < nx, y < ny the linear taper over the padding layers, the cyclic
 * forward difference (Wavelet1D FIRSTORDERFORWARDDIFF,
 * src/wavelet1D.cpp:420-440), the unnormalised spectrum times conj(W(k))
 * for k <= nzp/2 (getCAmp(k, 1), src/wavelet.cpp:327-385), and the
 * inverse transform scaled by 1/nzp (src/wavelet.cpp:264-280).  The 1-D
 * transforms here are double precision.                                */
/* ------------------------------------------------------------------ */
int orc_synt_seismic(int nxp, int nyp, int nzp, int nx, int ny, int nz, int ntheta,
                     const float *A, const float *wavelet, const float *const *m,
                     float *const *out) {
  int cnxp = nxp / 2 + 1, rnxp = 2 * cnxp, cnzp = nzp / 2 + 1;
  long plane = (long)rnxp * nyp, rsize = plane * nzp;
  float *imp = (float *)malloc(sizeof(float) * nzp), *dif = (float *)malloc(sizeof(float) * nzp);
  cd *W = (cd *)malloc(sizeof(cd) * nzp), *x = (cd *)malloc(sizeof(cd) * nzp);
  if (nz < 1 || nz > nzp || nx > nxp || ny > nyp) return 1;
  for (int l = 0; l < ntheta; ++l) {
    const float *a = A + 3 * l;
    for (int k = 0; k < nzp; ++k) { W[k].re = wavelet[(long)l * nzp + k]; W[k].im = 0.0; }
    dft1d(W, nzp, -1);
    float *o = out[l];
    for (long c = 0; c < rsize; ++c) {
      float v = 0.0f;
      v += m[0][c] * a[0];
      v += m[1][c] * a[1];
      v += m[2][c] * a[2];
      o[c] = v;
    }
    for (int i = 0; i < nx; ++i)
      for (int j = 0; j < ny; ++j) {
        long t = i + (long)rnxp * j;
        int k;
        for (k = 0; k < nz; ++k) imp[k] = o[t + k * plane];
        float fac = 1.0f / (float)(nzp - nz - 1);
        for (; k < nzp; ++k) imp[k] = fac * ((float)(k - nz) * imp[0] + (float)(nzp - k - 1) * imp[nz - 1]);
        for (k = 0; k < nzp; ++k) dif[k] = (k == nzp - 1) ? imp[0] - imp[k] : imp[k + 1] - imp[k];
        for (k = 0; k < nzp; ++k) { x[k].re = dif[k]; x[k].im = 0.0; }
        dft1d(x, nzp, -1);
        for (k = 0; k < cnzp; ++k) {
          cd r = x[k], w = W[k], sv;
          sv.re = r.re * w.re + r.im * w.im;
          sv.im = -r.re * w.im + r.im * w.re;
          x[k] = sv;
        }
        /* Hermitian completion of the half spectrum, as a c2r transform
         * reads it (imaginary parts of k = 0 and nzp/2 dropped) */
        x[0].im = 0.0;
        if (nzp % 2 == 0) x[nzp / 2].im = 0.0;
        for (k = cnzp; k < nzp; ++k) { x[k].re = x[nzp - k].re; x[k].im = -x[nzp - k].im; }
        dft1d(x, nzp, +1);
        for (k = 0; k < nzp; ++k) o[t + k * plane] = (float)(x[k].re / (double)nzp);
      }
  }
  free(imp); free(dif); free(W); free(x);
  return 0;
}

/* ------------------------------------------------------------------ */
/* Prior and noise correlation grids.                                   */
/* computeCircCorrT + makeCircCorrTPosDef                               */
/* (src/seismicparametersholder.cpp:430-499); transforms in double.     */
/* ------------------------------------------------------------------ */
int orc_circ_corr_t(const float *prior_corr_t, int n, int low_int_cut, int nzp,
                    float *circ_corr_t) {
  int cn = nzp / 2 + 1;
  cd *x = (cd *)malloc(sizeof(cd) * nzp);
  if (!prior_corr_t || n < 1 || prior_corr_t[0] == 0.0f) { free(x); return 1; }
  for (int k = 0; k < nzp; ++k) {
    int refk = k < cn ? k : nzp - k;
    x[k].re = refk < n ? prior_corr_t[refk] : 0.0;
    x[k].im = 0.0;
  }
  dft1d(x, nzp, -1);
  for (int k = 0; k < cn; ++k) {
    double m = k <= low_int_cut ? 0.0 : (double)(float)sqrt(x[k].re * x[k].re + x[k].im * x[k].im);
    x[k].re = m; x[k].im = 0.0;
  }
  for (int k = cn; k < nzp; ++k) x[k] = x[nzp - k];
  dft1d(x, nzp, +1);
  if (!((float)x[0].re > 1.e-5f)) { free(x); return 1; }
  float scale = 1.0f / (float)x[0].re;
  for (int k = 0; k < nzp; ++k) circ_corr_t[k] = (float)x[k].re * scale;
  free(x);
  return 0;
}

/* cycleI / cycleJ of src/fftgrid.cpp:1082-1087 and :1130-1135 */
static int cyc(int i, int n) {
  int c = i - n;
  if (i < -c) c = i;
  return c;
}

/* FFTGrid::fillInParamCorr (src/fftgrid.cpp:1118-1164), then
 * multiplyByScalar(float(var0_pq)) over every cell (:1992-2000) as
 * SeismicParametersHolder::initializeCorrelations does (:196-221). */
int orc_fill_prior_cov(int nxp, int nyp, int nzp, const float *corr_xy,
                       const float *circ, float gradI, float gradJ,
                       const double *var0, float *const *cov) {
  int rnxp = 2 * (nxp / 2 + 1);
  const int pq[6][2] = {{0, 0}, {1, 1}, {2, 2}, {0, 1}, {0, 2}, {1, 2}};
  long idx = 0;
  for (int k = 0; k < nzp; ++k)
    for (int j = 0; j < nyp; ++j)
      for (int i = 0; i < rnxp; ++i, ++idx) {
        float value;
        if (i < nxp) {
          int cycleI = cyc(i, nxp), cycleJ = cyc(j, nyp);
          float subK = k + cycleI * gradI + cycleJ * gradJ;
          int baseK = (int)floorf(subK);
          subK -= baseK;
          while (baseK < 0) baseK += nzp;
          while (baseK >= nzp) baseK -= nzp;
          value = (1 - subK) * circ[baseK];
          if (baseK != nzp - 1) value += subK * circ[baseK + 1];
          else value += subK * circ[0];
          value *= corr_xy[i + nxp * j];
        } else {
          value = -99999.0f; /* RMISSING */
        }
        for (int t = 0; t < 6; ++t) cov[t][idx] = value * (float)var0[3 * pq[t][0] + pq[t][1]];
      }
  return 0;
}

/* FFTGrid::fillInErrCorr (src/fftgrid.cpp:1064-1116). */
int orc_fill_err_corr(int nxp, int nyp, int nzp, const float *corr_xy,
                      float gradI, float gradJ, float *err) {
  int rnxp = 2 * (nxp / 2 + 1), range = 1;
  long idx = 0;
  for (int k = 0; k < nzp; ++k)
    for (int j = 0; j < nyp; ++j)
      for (int i = 0; i < rnxp; ++i, ++idx) {
        int cycleI = cyc(i, nxp), cycleJ = cyc(j, nyp);
        float subK = k + cycleI * gradI + cycleJ * gradJ;
        float value;
        if (i < nxp) {
          if (fabsf(subK) < range * 1.0f || fabsf(subK - nzp) < range * 1.0f) {
            int baseK = (int)subK;
            subK -= baseK;
            while (baseK < -range) baseK += nzp;
            while (baseK >= range) baseK -= nzp;
            if (baseK < 0) { baseK = -1 - baseK; subK = 1 - subK; }
            value = (1 - subK) * corr_xy[i + nxp * j];
          } else {
            value = 0;
          }
        } else {
          value = -99999.0f;
        }
        err[idx] = value;
      }
  return 0;
}

/* ------------------------------------------------------------------ */
/* Time-lapse state: State4D (src/state4d.cpp)                          */
/* ------------------------------------------------------------------ */
/* (p, q) of State4D's upper-triangle order and the same entry's slot in
 * the posterior's covariance order. */
static const int s4_p[6] = {0, 0, 0, 1, 1, 2}, s4_q[6] = {0, 1, 2, 1, 2, 2};
static const int s4_unit[6] = {0, 3, 4, 1, 5, 2};

static cf ld_cf(const float *g, long long b) { cf v = {g[2 * b], g[2 * b + 1]}; return v; }
static void st_cf(float *g, long long b, cf v) { g[2 * b] = v.re; g[2 * b + 1] = v.im; }
static cf conj_cf(cf a) { cf v = {a.re, -a.im}; return v; }

/* The full 6x6 prior of one bin: upper triangle from the grids, lower as
 * its conjugate (src/state4d.cpp:203-225 and :341-380). */
static void s4_full(long long b, const float *const *ss, const float *const *dd,
                    const float *const *sd, cf F[6][6]) {
  for (int r = 0; r < 6; ++r) {
    F[s4_p[r]][s4_q[r]] = ld_cf(ss[r], b);
    F[s4_p[r] + 3][s4_q[r] + 3] = ld_cf(dd[r], b);
  }
  for (int l = 0; l < 3; ++l)
    for (int m = 0; m < 3; ++m) F[l][m + 3] = ld_cf(sd[3 * l + m], b);
  for (int l = 0; l < 6; ++l)
    for (int m = l + 1; m < 6; ++m) F[m][l] = conj_cf(F[l][m]);
}

/* State4D::merge (src/state4d.cpp:90-159) and mergeCov (:161-249). */
void orc_state4d_merge(long long n, const float *const *ms, const float *const *md,
                       const float *const *ss, const float *const *dd,
                       const float *const *sd, float *const *mu, float *const *cov) {
  for (long long b = 0; b < n; ++b) {
    if (mu)
      for (int l = 0; l < 3; ++l) {
        cf s = ld_cf(ms[l], b), d = ld_cf(md[l], b), v = {s.re + d.re, s.im + d.im};
        st_cf(mu[l], b, v);
      }
    cf F[6][6];
    s4_full(b, ss, dd, sd, F);
    for (int r = 0; r < 6; ++r) {
      int l = s4_p[r], m = s4_q[r];
      cf v;
      v.re = F[l][m].re; v.re += F[l + 3][m + 3].re; v.re += F[l + 3][m].re; v.re += F[l][m + 3].re;
      v.im = F[l][m].im; v.im += F[l + 3][m + 3].im; v.im += F[l + 3][m].im; v.im += F[l][m + 3].im;
      st_cf(cov[s4_unit[r]], b, v);
    }
  }
}

/* lib_matrAXeqBMatCpx (libs/lib/lib_matr.c:330-365) for an n x nc matrix B
 * stored row-major with leading dimension ldb. */
static void axeqb_fw(int n, cf L[][ORC_MAXT], cf *B, int ldb, int nc) {
  cf lx; float help;
  for (int c = 0; c < nc; ++c) {
    for (int i = 0; i < n; ++i) {
      lx = B[i * ldb + c];
      for (int j = 0; j < i; ++j) {
        lx.re -= (B[j * ldb + c].re * L[i][j].re - B[j * ldb + c].im * L[i][j].im);
        lx.im -= (B[j * ldb + c].im * L[i][j].re + B[j * ldb + c].re * L[i][j].im);
      }
      help = (L[i][i].re * L[i][i].re + L[i][i].im * L[i][i].im);
      B[i * ldb + c].re = (lx.re * L[i][i].re + lx.im * L[i][i].im) / help;
      B[i * ldb + c].im = (lx.im * L[i][i].re - lx.re * L[i][i].im) / help;
    }
    for (int i = n - 1; i >= 0; --i) {
      lx = B[i * ldb + c];
      for (int j = n - 1; j > i; --j) {
        lx.re = lx.re - (B[j * ldb + c].re * L[j][i].re + B[j * ldb + c].im * L[j][i].im);
        lx.im = lx.im - (-B[j * ldb + c].re * L[j][i].im + B[j * ldb + c].im * L[j][i].re);
      }
      help = (L[i][i].re * L[i][i].re + L[i][i].im * L[i][i].im);
      B[i * ldb + c].re = (lx.re * L[i][i].re - lx.im * L[i][i].im) / help;
      B[i * ldb + c].im = (lx.im * L[i][i].re + lx.re * L[i][i].im) / help;
    }
  }
}

/* x += a b in lib_matrProdCpx's form (libs/lib/lib_matr.c:548-566). */
static void cmac_f(cf *x, cf a, cf b) {
  x->re += a.re * b.re - a.im * b.im;
  x->im += a.im * b.re + a.re * b.im;
}

/* State4D::split (src/state4d.cpp:251-525).  Returns the bins whose 3x3
 * Cholesky failed (prior kept). */
long long orc_state4d_split(long long n, float *const *ms, float *const *md,
                            float *const *ss, float *const *dd, float *const *sd,
                            const float *const *mu, const float *const *cov) {
  long long fails = 0;
  for (long long b = 0; b < n; ++b) {
    cf F[6][6], muF[6], muP[3], SP[3][3], muC[3], FvC[6][3], SC[3][3];
    cf L[ORC_MAXT][ORC_MAXT], B[3][6];
    s4_full(b, (const float *const *)ss, (const float *const *)dd,
            (const float *const *)sd, F);
    for (int l = 0; l < 3; ++l) { muF[l] = ld_cf(ms[l], b); muF[l + 3] = ld_cf(md[l], b); }
    for (int l = 0; l < 3; ++l) muP[l] = ld_cf(mu[l], b);
    for (int r = 0; r < 6; ++r) {
      cf v = ld_cf(cov[s4_unit[r]], b);
      SP[s4_p[r]][s4_q[r]] = v;
      SP[s4_q[r]][s4_p[r]] = v; /* copied, not conjugated (:370-372) */
    }
    for (int l = 0; l < 3; ++l) {
      muC[l].re = muF[l].re + muF[l + 3].re;
      muC[l].im = muF[l].im + muF[l + 3].im;
    }
    for (int l = 0; l < 6; ++l)
      for (int m = 0; m < 3; ++m) {
        FvC[l][m].re = F[l][m].re + F[l][m + 3].re;
        FvC[l][m].im = F[l][m].im + F[l][m + 3].im;
      }
    for (int l = 0; l < 3; ++l)
      for (int m = 0; m < 3; ++m) {
        SC[l][m].re = FvC[l][m].re + FvC[l + 3][m].re;
        SC[l][m].im = FvC[l][m].im + FvC[l + 3][m].im;
        L[l][m] = SC[l][m];
      }
    for (int l = 0; l < 6; ++l)
      for (int m = 0; m < 3; ++m) B[m][l] = conj_cf(FvC[l][m]);
    if (chol_f(3, L) == 0) {
      cf H[3][6], P[6][6], muFP[6];
      axeqb_fw(3, L, &B[0][0], 6, 6);
      for (int l = 0; l < 3; ++l)
        for (int m = 0; m < 3; ++m) { SP[l][m].re -= SC[l][m].re; SP[l][m].im -= SC[l][m].im; }
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 6; ++j) {
          cf x = {0.0f, 0.0f};
          for (int k = 0; k < 3; ++k) cmac_f(&x, SP[i][k], B[k][j]);
          H[i][j] = x;
        }
      for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) {
          cf x = {0.0f, 0.0f};
          for (int k = 0; k < 3; ++k) cmac_f(&x, conj_cf(B[k][i]), H[k][j]);
          P[i][j] = x;
        }
      for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) { P[i][j].re += F[i][j].re; P[i][j].im += F[i][j].im; }
      for (int l = 0; l < 3; ++l) { muP[l].re -= muC[l].re; muP[l].im -= muC[l].im; }
      for (int i = 0; i < 6; ++i) {
        cf x = {0.0f, 0.0f};
        for (int k = 0; k < 3; ++k) cmac_f(&x, conj_cf(B[k][i]), muP[k]);
        muFP[i] = x;
      }
      for (int i = 0; i < 6; ++i) { muFP[i].re += muF[i].re; muFP[i].im += muF[i].im; }
      memcpy(F, P, sizeof F);
      memcpy(muF, muFP, sizeof muF);
    } else {
      ++fails;
    }
    for (int r = 0; r < 6; ++r) {
      st_cf(ss[r], b, F[s4_p[r]][s4_q[r]]);
      st_cf(dd[r], b, F[s4_p[r] + 3][s4_q[r] + 3]);
    }
    for (int l = 0; l < 3; ++l)
      for (int m = 0; m < 3; ++m) st_cf(sd[3 * l + m], b, F[l][m + 3]);
    for (int l = 0; l < 3; ++l) { st_cf(ms[l], b, muF[l]); st_cf(md[l], b, muF[l + 3]); }
  }
  return fails;
}

/* State4D::evolve (src/state4d.cpp:527-730): double arithmetic (the
 * reference's FLENS matrices), each product-sum a chain of fused
 * multiply-adds in natural order (C99 fma, correctly rounded), one rounding
 * to float.  Both parts of the 6x6 matrix are mirrored unchanged
 * (:660-690). */
void orc_state4d_evolve(long long n, float *const *ms, float *const *md,
                        float *const *ss, float *const *dd, float *const *sd,
                        const double *E, const double *cm, const double *cc,
                        const float *lambda, float zero_scale) {
  for (long long b = 0; b < n; ++b) {
    double lam = (double)lambda[2 * b];
    float sc = b == 0 ? zero_scale : 0.0f;
    double mr[6], mi[6], Sr[6][6], Si[6][6], Tr[6][6], Ti[6][6];
    for (int l = 0; l < 3; ++l) {
      cf s = ld_cf(ms[l], b), d = ld_cf(md[l], b);
      mr[l] = s.re; mi[l] = s.im; mr[l + 3] = d.re; mi[l + 3] = d.im;
    }
    for (int d = 0; d < 6; ++d) {
      double xr = 0.0, xi = 0.0;
      for (int e = 0; e < 6; ++e) { xr = fma(E[6 * d + e], mr[e], xr); xi = fma(E[6 * d + e], mi[e], xi); }
      xr = fma(cm[d], (double)sc, xr);
      cf v = {(float)xr, (float)xi};
      st_cf(d < 3 ? ms[d] : md[d - 3], b, v);
    }
    for (int r = 0; r < 6; ++r) {
      int p = s4_p[r], q = s4_q[r];
      cf s = ld_cf(ss[r], b), d = ld_cf(dd[r], b);
      Sr[p][q] = Sr[q][p] = s.re; Si[p][q] = Si[q][p] = s.im;
      Sr[p + 3][q + 3] = Sr[q + 3][p + 3] = d.re; Si[p + 3][q + 3] = Si[q + 3][p + 3] = d.im;
    }
    for (int l = 0; l < 3; ++l)
      for (int m = 0; m < 3; ++m) {
        cf v = ld_cf(sd[3 * l + m], b);
        Sr[l][m + 3] = Sr[m + 3][l] = v.re;
        Si[l][m + 3] = Si[m + 3][l] = v.im;
      }
    for (int i = 0; i < 6; ++i)
      for (int j = 0; j < 6; ++j) {
        double xr = 0.0, xi = 0.0;
        for (int k = 0; k < 6; ++k) { xr = fma(E[6 * i + k], Sr[k][j], xr); xi = fma(E[6 * i + k], Si[k][j], xi); }
        Tr[i][j] = xr; Ti[i][j] = xi;
      }
    for (int i = 0; i < 6; ++i)
      for (int j = i; j < 6; ++j) {
        double xr = 0.0, xi = 0.0;
        for (int k = 0; k < 6; ++k) { xr = fma(Tr[i][k], E[6 * j + k], xr); xi = fma(Ti[i][k], E[6 * j + k], xi); }
        xr = fma(cc[6 * i + j], lam, xr);
        cf v = {(float)xr, (float)xi};
        if (j < 3) {
          for (int r = 0; r < 6; ++r) if (s4_p[r] == i && s4_q[r] == j) st_cf(ss[r], b, v);
        } else if (i < 3) {
          st_cf(sd[3 * i + j - 3], b, v);
        } else {
          for (int r = 0; r < 6; ++r) if (s4_p[r] == i - 3 && s4_q[r] == j - 3) st_cf(dd[r], b, v);
        }
      }
  }
}

/* FFTGrid::fillInGenExpCorr (src/fftgrid.cpp:1167-1210). */
int orc_fill_gen_exp_corr(int nxp, int nyp, int nzp, double Rx, double Ry, double Rz,
                          float gradI, float gradJ, float *out) {
  int rnxp = 2 * (nxp / 2 + 1);
  long idx = 0;
  for (int k = 0; k < nzp; ++k)
    for (int j = 0; j < nyp; ++j)
      for (int i = 0; i < rnxp; ++i, ++idx) {
        float value;
        if (i < nxp) {
          int cycleI = cyc(i, nxp), cycleJ = cyc(j, nyp);
          float subK = k + cycleI * gradI + cycleJ * gradJ;
          while (subK < -nzp / 2.0) subK += nzp;
          while (subK >= nzp / 2.0) subK -= nzp;
          double qDist = (float)(cycleI * cycleI) / (Rx * Rx) + (cycleJ * cycleJ) / (Ry * Ry) +
                         (subK * subK) / (Rz * Rz);
          double dist = sqrt(qDist);
          value = (float)exp(-3.0 * dist);
        } else {
          value = -99999.0f; /* RMISSING */
        }
        out[idx] = value;
      }
  return 0;
}

/* ------------------------------------------------------------------ */
/* Data divided by the local scale wavelet                              */
/* ------------------------------------------------------------------ */
/* Real inverse of a half spectrum (FFTW's complex_to_real: the imaginary
 * parts of bin 0 and of bin n/2 are not read), unnormalised. */
static void real_inverse(const cf *h, int n, float *out, double scale) {
  cd *line = (cd *)malloc(sizeof(cd) * n);
  int c = n / 2 + 1;
  for (int k = 0; k < c; ++k) { line[k].re = h[k].re; line[k].im = h[k].im; }
  line[0].im = 0.0;
  if (n % 2 == 0) line[n / 2].im = 0.0;
  for (int k = c; k < n; ++k) { line[k].re = h[n - k].re; line[k].im = -h[n - k].im; }
  dft1d(line, n, +1);
  for (int i = 0; i < n; ++i) out[i] = (float)(line[i].re * scale);
  free(line);
}

/* FFTGrid::getDistToBoundary (src/fftgrid.cpp:1374-1414), i < np. */
static float dist_to_boundary(int i, int n, int np) {
  if (i < n) return 0.0f;
  float taper = (float)((n < np - n ? n : np - n) / 2.1);
  int below = np - i, above = i - (n - 1);
  return above < below ? (float)(above / taper) : (float)(below / taper);
}

/* The simbox index of a padded trace (src/crava.cpp:622-640). */
static int mirror_index(int i, int n, int np) {
  if (i > 3 * n - 1) i = 0;
  if (i > (np + n) / 2) i = np - i;
  if (i >= n) i = 2 * n - i - 1;
  return i;
}

/* Wavelet::findNormWithinFrequencyBand (src/wavelet.cpp:811-833). */
static float band_norm(const cf *c, int nzp, float dz, float lo, float hi) {
  int cnzp = nzp / 2 + 1;
  float dOmega = (float)(1.0 / (nzp * dz * 0.001));
  int loI = (int)floorf(lo / dOmega), hiI = (int)ceilf(hi / dOmega);
  if (loI < 0) loI = 0;
  if (hiI > cnzp) hiI = cnzp;
  double fac = 1.0 / (double)nzp, norm2 = 0.0;
  for (int i = loI; i < hiI; ++i) norm2 += (double)(2.0 * fac * (c[i].re * c[i].re + c[i].im * c[i].im));
  if (loI == 0) norm2 -= fac * (c[0].re * c[0].re + c[0].im * c[0].im);
  return (float)sqrt(norm2);
}

/* Crava::divideDataByScaleWavelet (src/crava.cpp:591-722) with
 * computeAdjustmentFactor (:725-817), 1-D wavelets, without the closing
 * interpolateSeismic: per trace the local wavelet (shiftAndScale,
 * src/wavelet1D.cpp:539-561) goes back to the time domain, its
 * difference wavelets (:420-479) and spectra are formed, and the trace's
 * in-band bins are multiplied by the adjustment factor. */
int orc_divide_data(const crava_oracle_params *p, float *const *data, const float *cov_col,
                    const double *rel_thick, int nx, int ny, float dz, const float *shift,
                    const float *gain) {
  const int nxp = p->nxp, nyp = p->nyp, nzp = p->nzp, nt = p->ntheta, nz = p->nz;
  const int cnzp = nzp / 2 + 1, rnxp = 2 * (nxp / 2 + 1);
  const float RM = -99999.0f, tolFac = 0.05f;
  float *w = (float *)malloc(sizeof(float) * nzp), *r = (float *)malloc(sizeof(float) * nzp);
  float *wl = (float *)malloc(sizeof(float) * nzp), *e1 = (float *)malloc(sizeof(float) * nzp);
  float *e2 = (float *)malloc(sizeof(float) * nzp), *e3 = (float *)malloc(sizeof(float) * nzp);
  float *tr = (float *)malloc(sizeof(float) * nzp);
  cf *W = (cf *)malloc(sizeof(cf) * cnzp), *Wl = (cf *)malloc(sizeof(cf) * cnzp);
  cf *E3 = (cf *)malloc(sizeof(cf) * cnzp), *R = (cf *)malloc(sizeof(cf) * cnzp);
  cf *D = (cf *)malloc(sizeof(cf) * cnzp), *adj = (cf *)malloc(sizeof(cf) * cnzp);
  const float sq = (float)sqrtf((float)nzp);
  for (int l = 0; l < nt; ++l) {
    memcpy(w, p->wavelet + (size_t)l * nzp, sizeof(float) * nzp);
    const float wn = p->wavelet_norm ? p->wavelet_norm[l] : time_norm(w, nzp);
    real_spectrum(w, nzp, W);
    /* rcCovT: computeReflectionCoefficientTimeCovariance (:476-508) on
     * getPriorCorrTFiltered (src/seismicparametersholder.cpp:504-530) */
    double eiVar = 0.0;
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b)
        eiVar += p->A[3 * l + a] * (float)p->var0[3 * a + b] * p->A[3 * l + b];
    float constant = cov_col[0];
    for (int i = 0; i < nzp; ++i) {
      int refk = i < nzp / 2 + 1 ? i : nzp - i;
      float corr = refk < nz ? cov_col[refk] / constant : 0.0f;
      r[i] = (float)(eiVar * corr);
    }
    {
      float first = r[0], prev = r[nzp - 1];
      for (int i = 0; i < nzp - 1; ++i) {
        float curr = r[i], next = r[i + 1];
        r[i] = 2 * curr - next - prev;
        prev = curr;
      }
      r[nzp - 1] = 2 * r[nzp - 1] - first - prev;
    }
    real_spectrum(r, nzp, R);
    float modW = wn;
    modW *= modW;
    float maxfrequency = (float)((nzp / 2) * 1000.0 * nz) / (float)(p->lz * nzp);
    modW *= maxfrequency / p->high_cut;
    const float errorVar = (float)p->theta_cov[l * nt + l];
    for (int j = 0; j < nyp; ++j)
      for (int i = 0; i < nxp; ++i) {
        int iInd = mirror_index(i, nx, nxp), jInd = mirror_index(j, ny, nyp);
        /* the local wavelet: shiftAndScale of the spectrum, then back to
         * the time domain (the Wavelet(wavelet, difftype) constructor) */
        float ts = 0.0f, g = 1.0f;
        /* getLocalTimeshift / getLocalGainFactor: only inside the grids
         * (src/wavelet.cpp:1143-1172) */
        if (iInd >= 0 && iInd < nx && jInd >= 0 && jInd < ny) {
          size_t o = (size_t)l * nx * ny + iInd + (size_t)nx * jInd;
          if (shift && shift[o] != -999.0f) ts = shift[o];
          if (gain && gain[o] != -999.0f) g = gain[o];
        }
        float iShift = ts / dz;
        for (int k = 0; k < cnzp; ++k) {
          cf am, t;
          am.re = (float)(g * cos(2.0 * (3.14159265358979323846 * (iShift) * k) / (float)nzp));
          am.im = (float)(g * sin(-2.0 * (3.14159265358979323846 * (iShift) * k) / (float)nzp));
          t.re = am.re * W[k].re - am.im * W[k].im;
          t.im = am.im * W[k].re + am.re * W[k].im;
          Wl[k] = t;
        }
        real_inverse(Wl, nzp, wl, 1.0 / (double)nzp);
        for (int n = 0; n < nzp; ++n) e1[n] = (n == nzp - 1) ? wl[0] - wl[n] : wl[n + 1] - wl[n];
        for (int n = 0; n < nzp; ++n) e2[n] = (n == 0) ? e1[0] - e1[nzp - 1] : e1[n] - e1[n - 1];
        for (int n = 0; n < nzp; ++n) {
          float d = (n == 0) ? e2[1] - e2[nzp - 1] : (n == nzp - 1) ? e2[0] - e2[n - 1] : e2[n + 1] - e2[n - 1];
          e3[n] = (float)(0.5 * d);
        }
        real_spectrum(e3, nzp, E3);
        {
          float inv = 1.0f / band_norm(E3, nzp, dz, p->low_cut, p->high_cut);
          float *f = (float *)E3; /* multiplyRAmpByConstant: floats past nzp RMISSING */
          for (int q = 0; q < 2 * cnzp; ++q) f[q] = q < nzp ? f[q] * inv : RM;
        }
        real_spectrum(wl, nzp, Wl); /* wLocal->fft1DInPlace() */
        double relT = rel_thick[i + (size_t)nxp * j];
        float sf = (float)(relT * 1.0f);
        for (int k = 0; k < cnzp; ++k) {
          cf wLoc = get_camp_scaled(Wl, nzp, k, sf);
          float wLoc2 = wLoc.re * wLoc.re + wLoc.im * wLoc.im;
          cf wGlob = W[k];
          float wGlob2 = wGlob.re * wGlob.re + wGlob.im * wGlob.im;
          cf v = wLoc;
          float sizeLoc = (v.re * v.re + v.im * v.im) / (wn * wn);
          v = get_camp_scaled(E3, nzp, k, sf);
          sizeLoc += v.re * v.re + v.im * v.im;
          v = Wl[k];
          float sizeGlob = (v.re * v.re + v.im * v.im) / (wn * wn);
          v = E3[k];
          sizeGlob += v.re * v.re + v.im * v.im;
          float sigma2Loc = errorVar * (p->wnc + (1.0f - p->wnc) * 0.5f * sizeLoc);
          float sigma2Glob = errorVar * (p->wnc + (1.0f - p->wnc) * 0.5f * sizeGlob);
          float tau2 = fabsf(R[k].re);
          float wGlob2Adj = wGlob2, wLoc2Adj = wLoc2;
          if (wGlob2 < tolFac * modW) wGlob2Adj = (float)(0.5f * (wGlob2 + tolFac * modW));
          if (wLoc2 < tolFac * modW) wLoc2Adj = (float)(0.5f * (wLoc2 + tolFac * modW));
          if (wLoc2Adj < tolFac * wGlob2Adj) {
            wLoc2Adj = (float)(0.5f * (wLoc2 + tolFac * wGlob2Adj));
            sigma2Loc *= wLoc2Adj / wLoc2;
          }
          adj[k].re = (wLoc.re / (tau2 * wLoc2Adj + sigma2Loc)) / (wGlob2Adj / (tau2 * wGlob2 + sigma2Glob));
          adj[k].im = (wLoc.im / (tau2 * wLoc2Adj + sigma2Loc)) / (wGlob2Adj / (tau2 * wGlob2 + sigma2Glob));
        }
        /* the trace: taper, transform, adjust in band, transform back */
        float *g0 = data[l] + i + (size_t)rnxp * j;
        for (int k = 0; k < nzp; ++k) {
          tr[k] = g0[(size_t)rnxp * nyp * k] / sq;
          if (k > nz) {
            float dist = dist_to_boundary(k, nz, nzp);
            float m = 1 - dist * dist;
            tr[k] *= m > 0.0f ? m : 0.0f;
          }
        }
        real_spectrum(tr, nzp, D);
        double deltaF = (double)nz * 1000.0 / (relT * p->lz * (double)nzp);
        for (int k = 0; k < cnzp; ++k) {
          if ((deltaF * k < p->high_cut) && (deltaF * k > p->low_cut)) {
            float tmp = D[k].re * adj[k].re - D[k].im * adj[k].im;
            D[k].im = D[k].im * adj[k].re + D[k].re * adj[k].im;
            D[k].re = tmp;
          } else {
            D[k].re = 0.0f; D[k].im = 0.0f;
          }
        }
        real_inverse(D, nzp, tr, 1.0);
        for (int k = 0; k < nzp; ++k) g0[(size_t)rnxp * nyp * k] = tr[k] / sq;
      }
  }
  free(w); free(r); free(wl); free(e1); free(e2); free(e3); free(tr);
  free(W); free(Wl); free(E3); free(R); free(D); free(adj);
  return 0;
}

/* ------------------------------------------------------------------ */
/* Low-energy traces: FFTGrid::interpolateSeismic                       */
/* ------------------------------------------------------------------ */
typedef struct { float *g; int nx, ny, nz, nxp, nyp, nzp, rnxp; short *flags; } orc_interp;

static float *orc_at(const orc_interp *s, int i, int j, int k) {
  return s->g + i + (size_t)s->rnxp * (j + (size_t)s->nyp * k);
}

/* FFTGrid::interpolateTrace (src/fftgrid.cpp:2658-2695) */
static int orc_interp_trace(orc_interp *s, int index, int i, int j) {
  int nx = s->nx, ny = s->ny, nt = 0;
  int left = i > 0 && (s->flags[index - 1] % 2) == 0;
  int right = i < nx - 1 && (s->flags[index + 1] % 2) == 0;
  int up = j > 0 && (s->flags[index - nx] % 2) == 0;
  int down = j < ny - 1 && (s->flags[index + nx] % 2) == 0;
  nt = left + right + up + down;
  if (nt > 1) {
    float *mean = (float *)malloc(sizeof(float) * s->nzp);
    for (int k = 0; k < s->nzp; ++k) mean[k] = left ? *orc_at(s, i - 1, j, k) : 0.0f;
    if (right) for (int k = 0; k < s->nzp; ++k) mean[k] += *orc_at(s, i + 1, j, k);
    if (up) for (int k = 0; k < s->nzp; ++k) mean[k] += *orc_at(s, i, j - 1, k);
    if (down) for (int k = 0; k < s->nzp; ++k) mean[k] += *orc_at(s, i, j + 1, k);
    for (int k = 0; k < s->nzp; ++k) *orc_at(s, i, j, k) = mean[k] / (float)nt;
    free(mean);
    s->flags[index]--;
  }
  return s->flags[index];
}

/* FFTGrid::getFillNumber (src/fftgrid.cpp:1319-1357), i < np */
static int orc_fill_number(int i, int n, int np) {
  if (i < n) return i;
  int below = np - i - 1, above = i - n + 1;
  if (above < below) return n - above > n / 2 ? n - above : n / 2;
  return below < n / 2 ? below : n / 2;
}

/* FFTGrid::interpolateSeismic (src/fftgrid.cpp:2564-2654) and
 * extrapolateSeismic (:2699-2731) on one real padded data grid. */
int orc_interpolate_seismic(float *grid, int nxp, int nyp, int nzp, int nx, int ny, int nz,
                            float energy_threshold, int *n_interpolated, int *n_zero) {
  orc_interp s = {grid, nx, ny, nz, nxp, nyp, nzp, 2 * (nxp / 2 + 1), NULL};
  short *flags = (short *)malloc(sizeof(short) * nx * ny);
  float *energyMap = (float *)malloc(sizeof(float) * nx * ny);
  s.flags = flags;
  int flag = 0, imin = nx, imax = 0, jmin = ny, jmax = 0, index = 0;
  float totalEnergy = 0;
  for (int j = 0; j < ny; j++)
    for (int i = 0; i < nx; i++) {
      float energy = 0;
      for (int k = 0; k < nz; k++) {
        float value = *orc_at(&s, i, j, k);
        energy += value * value;
      }
      energyMap[index] = energy;
      totalEnergy += energy;
      index++;
    }
  index = 0;
  float energyLimit = energy_threshold * totalEnergy / (float)(nx * ny);
  int nInter = 0, nInter0 = 0;
  for (int j = 0; j < ny; j++)
    for (int i = 0; i < nx; i++) {
      int curFlag = 0;
      if (energyMap[index] <= energyLimit) {
        curFlag = 1;
        nInter++;
        if (energyMap[index] == 0.0f) nInter0++;
      }
      flags[index] = (short)(flag + curFlag);
      if (curFlag == 1) flag = 2;
      else {
        if (i < imin) imin = i;
        if (i > imax) imax = i;
        if (j < jmin) jmin = j;
        if (j > jmax) jmax = j;
      }
      index++;
    }
  int curIndex = 0;
  for (int j = 0; j < ny; j++)
    for (int i = 0; i < nx; i++) {
      if ((flags[curIndex] % 2) == 1) {
        if ((orc_interp_trace(&s, curIndex, i, j) % 2) == 0) {
          index = curIndex - 1;
          while (index >= 0 && flags[index] > 1) {
            if ((flags[index] % 2) == 1) orc_interp_trace(&s, index, index % nx, index / nx);
            index--;
          }
          if (index < 0) index = 0;
          index++;
          while (flags[index - 1] == 0 && index <= curIndex) {
            if (flags[index] > 1) flags[index] -= 2;
            index++;
          }
        }
      }
      curIndex++;
    }
  if (imin <= imax && jmin <= jmax) {
    for (int j = 0; j < nyp; j++) {
      int refj = orc_fill_number(j, ny, nyp);
      if (refj < jmin) refj = jmin; else if (refj > jmax) refj = jmax;
      for (int i = 0; i < nxp; i++) {
        if (i < imin || i > imax || j < jmin || j > jmax) {
          int refi = orc_fill_number(i, nx, nxp);
          if (refi < imin) refi = imin; else if (refi > imax) refi = imax;
          for (int k = 0; k < nzp; k++) {
            float value = *orc_at(&s, refi, refj, k);
            float distx = dist_to_boundary(i, nx, nxp), disty = dist_to_boundary(j, ny, nyp);
            float distz = dist_to_boundary(k, nz, nzp);
            double b = 1.0 - distx * distx - disty * disty - distz * distz;
            float mult = (float)pow(b > 0.0 ? b : 0.0, 3);
            *orc_at(&s, i, j, k) = mult * value;
          }
        }
      }
    }
  }
  if (n_interpolated) *n_interpolated = nInter;
  if (n_zero) *n_zero = nInter0;
  free(flags);
  free(energyMap);
  return 0;
}

/* Crava::multiplyDataByScaleWaveletAndWriteToFile (src/crava.cpp:819-885)
 * before the file write, on time-domain residual grids (the caller has
 * made the invFFTInPlace): each simbox trace times the conjugate of
 * getCAmp(k, sf) of its local wavelet. */
int orc_multiply_data(const crava_oracle_params *p, float *const *data, const double *rel_thick,
                      int nx, int ny, float dz, const float *shift, const float *gain) {
  const int nxp = p->nxp, nyp = p->nyp, nzp = p->nzp, nt = p->ntheta;
  const int cnzp = nzp / 2 + 1, rnxp = 2 * (nxp / 2 + 1);
  float *w = (float *)malloc(sizeof(float) * nzp), *tr = (float *)malloc(sizeof(float) * nzp);
  cf *W = (cf *)malloc(sizeof(cf) * cnzp), *Wl = (cf *)malloc(sizeof(cf) * cnzp);
  cf *D = (cf *)malloc(sizeof(cf) * cnzp);
  for (int l = 0; l < nt; ++l) {
    memcpy(w, p->wavelet + (size_t)l * nzp, sizeof(float) * nzp);
    real_spectrum(w, nzp, W);
    for (int i = 0; i < nx; ++i)
      for (int j = 0; j < ny; ++j) {
        float sf = (float)rel_thick[i + (size_t)nxp * j] * 1.0f;
        float *g0 = data[l] + i + (size_t)rnxp * j;
        for (int k = 0; k < nzp; ++k) tr[k] = g0[(size_t)rnxp * nyp * k] / (float)sqrtf((float)nzp);
        real_spectrum(tr, nzp, D);
        float ts = 0.0f, g = 1.0f;
        size_t o = (size_t)l * nx * ny + i + (size_t)nx * j;
        if (shift && shift[o] != -999.0f) ts = shift[o];
        if (gain && gain[o] != -999.0f) g = gain[o];
        float iShift = ts / dz;
        for (int k = 0; k < cnzp; ++k) {
          cf am, t;
          am.re = (float)(g * cos(2.0 * (3.14159265358979323846 * (iShift) * k) / (float)nzp));
          am.im = (float)(g * sin(-2.0 * (3.14159265358979323846 * (iShift) * k) / (float)nzp));
          t.re = am.re * W[k].re - am.im * W[k].im;
          t.im = am.im * W[k].re + am.re * W[k].im;
          Wl[k] = t;
        }
        for (int k = 0; k < cnzp; ++k) {
          cf sv = get_camp_scaled(Wl, nzp, k, sf);
          float tmp = D[k].re * sv.re + D[k].im * sv.im;
          D[k].im = D[k].im * sv.re - D[k].re * sv.im;
          D[k].re = tmp;
        }
        real_inverse(D, nzp, tr, 1.0);
        for (int k = 0; k < nzp; ++k) g0[(size_t)rnxp * nyp * k] = tr[k] / (float)sqrt((double)nzp);
      }
  }
  free(w); free(tr); free(W); free(Wl); free(D);
  return 0;
}
