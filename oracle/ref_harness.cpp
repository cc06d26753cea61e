/*
 * ref_harness.cpp -- drives the reference's own numerics, compiled from its
 * sources (FFTW 2.1.2 single precision, libs/lib/lib_matr.c,
 * libs/lib/random.cpp), in the order src/crava.cpp drives them.
 * TEST INFRASTRUCTURE ONLY: built by oracle/Makefile into oracle/_ref/ and
 * used to pin the restatement in crava_oracle.c and as the timed CPU
 * baseline.  src/crava.cpp itself cannot be compiled without a CBLAS, so
 * the per-bin loop below restates src/crava.cpp:1042-1151 while every
 * numerical call in it is the reference's own function.
 */
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "fftw.h"
#include "rfftw.h"
#include "lib/lib_matr.h"
#define private public /* read RandomGen's static state after a draw */
#include "lib/random.h"
#undef private

#include "crava_oracle.h"

/* random.cpp's file constructor links against NRLib::OpenRead; the harness
 * never calls it, so this minimal definition only satisfies the linker. */
namespace NRLib {
void OpenRead(std::ifstream &stream, const std::string &filename,
              std::ios_base::openmode mode) {
  stream.open(filename.c_str(), mode);
}
}  // namespace NRLib

namespace {

/* FFTGrid::multiplyByScalar, src/fftgrid.cpp:1992-2000 */
void multiply_by_scalar(float *g, long rsize, float s) {
  for (long i = 0; i < rsize; ++i) g[i] *= s;
}

fftw_complex **alloc_mat(int n1, int n2) {
  fftw_complex **m = new fftw_complex *[n1];
  for (int i = 0; i < n1; ++i) {
    m[i] = new fftw_complex[n2];
    std::memset(m[i], 0, sizeof(fftw_complex) * n2);
  }
  return m;
}
void free_mat(fftw_complex **m, int n1) {
  for (int i = 0; i < n1; ++i) delete[] m[i];
  delete[] m;
}

/* Wavelet::fft1DInPlace (src/wavelet.cpp:246-261) on a copy. */
std::vector<fftw_complex> spectrum1d(const float *w, int nzp) {
  int cnzp = nzp / 2 + 1;
  fftw_real *r = static_cast<fftw_real *>(fftw_malloc(2 * cnzp * sizeof(fftw_real)));
  for (int i = 0; i < 2 * cnzp; ++i) r[i] = i < nzp ? w[i] : 0.0f;
  rfftwnd_plan plan = rfftwnd_create_plan(1, &nzp, FFTW_REAL_TO_COMPLEX,
                                          FFTW_ESTIMATE | FFTW_IN_PLACE);
  rfftwnd_one_real_to_complex(plan, r, reinterpret_cast<fftw_complex *>(r));
  fftwnd_destroy_plan(plan);
  std::vector<fftw_complex> out(cnzp);
  std::memcpy(out.data(), r, sizeof(fftw_complex) * cnzp);
  fftw_free(r);
  return out;
}

/* Wavelet::getCAmp(k), src/wavelet.cpp:308-324 */
fftw_complex get_camp(const std::vector<fftw_complex> &c, int nzp, int k) {
  fftw_complex v;
  if (k < nzp / 2 + 1) { v.re = c[k].re; v.im = c[k].im; }
  else { v.re = c[nzp - k].re; v.im = -c[nzp - k].im; }
  return v;
}

/* Wavelet::getCAmp(k, scale), src/wavelet.cpp:327-385 */
fftw_complex get_camp_scaled(const std::vector<fftw_complex> &c, int nzp, int k, float scale) {
  const int cnzp = nzp / 2 + 1;
  fftw_complex value;
  float omega, dOmega;
  int omU, omL;
  const int refk = k < cnzp ? k : nzp - k;
  omega = float(refk) / scale;
  if (omega >= cnzp) {
    value.re = 0.0f;
    value.im = 0.0f;
  } else {
    omL = int(std::floor(omega));
    omU = int(std::floor(omega)) + 1;
    if (omU >= cnzp) omU -= 1;
    dOmega = omega - float(omL);
    value.re = c[omL].re * (1.0f - dOmega) + c[omU].re * dOmega;
    if (k < cnzp) value.im = (c[omL].im * (1.0f - dOmega) + c[omU].im * dOmega);
    else value.im = (-c[omL].im * (1.0f - dOmega) - c[omU].im * dOmega);
  }
  value.re /= scale;
  value.im /= scale;
  return value;
}

/* Wavelet::findNorm on a real wavelet, src/wavelet.cpp:789-808 */
float find_norm(const float *w, int n) {
  double norm2 = 0.0;
  for (int i = 0; i < n; ++i) norm2 += static_cast<double>(w[i] * w[i]);
  return static_cast<float>(std::sqrt(norm2));
}

struct KzTables {
  std::vector<fftw_complex> wd, e1, e2;
  std::vector<float> e3;
  std::vector<int> inv;
};

/* crava.cpp:952-976, 1024-1058 for the constant-thickness branch. */
void build_tables(const crava_oracle_params *p, KzTables &t) {
  const int nzp = p->nzp, nt = p->ntheta;
  std::vector<std::vector<fftw_complex>> W(nt), G(nt);
  std::vector<float> wn(nt), gn(nt);
  std::vector<float> e(nzp), f(nzp), g(nzp);
  for (int l = 0; l < nt; ++l) {
    const float *w = p->wavelet + static_cast<long>(l) * nzp;
    wn[l] = p->wavelet_norm ? p->wavelet_norm[l] : find_norm(w, nzp);
    W[l] = spectrum1d(w, nzp);
    /* Wavelet1D difference constructors, src/wavelet1D.cpp:420-479 */
    for (int i = 0; i < nzp; ++i) e[i] = (i == nzp - 1) ? w[0] - w[i] : w[i + 1] - w[i];
    for (int i = 0; i < nzp; ++i) f[i] = (i == 0) ? e[0] - e[nzp - 1] : e[i] - e[i - 1];
    for (int i = 0; i < nzp; ++i) {
      if (i == 0) g[i] = static_cast<fftw_real>(0.5 * (f[i + 1] - f[nzp - 1]));
      else if (i == nzp - 1) g[i] = static_cast<fftw_real>(0.5 * (f[0] - f[i - 1]));
      else g[i] = static_cast<fftw_real>(0.5 * (f[i + 1] - f[i - 1]));
    }
    gn[l] = find_norm(g.data(), nzp);
    G[l] = spectrum1d(g.data(), nzp);
  }
  /* Wavelet1D(FIRSTORDERFORWARDDIFF, nz, nzp), src/wavelet1D.cpp:368-394 */
  std::vector<float> d(nzp, 0.0f);
  d[0] = -1.0f; d[nzp - 1] = 1.0f;
  std::vector<fftw_complex> D = spectrum1d(d.data(), nzp);
  /* diff3Operator (src/crava.cpp:938-940): backward then central
   * difference of diff1Operator (src/wavelet1D.cpp:420-479) */
  std::vector<float> d2(nzp), d3(nzp);
  for (int i = 0; i < nzp; ++i) d2[i] = (i == 0) ? d[0] - d[nzp - 1] : d[i] - d[i - 1];
  for (int i = 0; i < nzp; ++i) {
    if (i == 0) d3[i] = static_cast<fftw_real>(0.5 * (d2[i + 1] - d2[nzp - 1]));
    else if (i == nzp - 1) d3[i] = static_cast<fftw_real>(0.5 * (d2[0] - d2[i - 1]));
    else d3[i] = static_cast<fftw_real>(0.5 * (d2[i + 1] - d2[i - 1]));
  }
  std::vector<fftw_complex> D3 = spectrum1d(d3.data(), nzp);

  t.wd.resize(static_cast<size_t>(nzp) * nt); t.e1.resize(t.wd.size());
  t.e2.resize(t.wd.size()); t.e3.resize(t.wd.size()); t.inv.resize(nzp);
  std::vector<fftw_complex> kW(nt);
  for (int k = 0; k < nzp; ++k) {
    float realFrequency = static_cast<float>((p->nz * 1000.0f) / (p->lz * nzp) * std::min(k, nzp - k));
    t.inv[k] = realFrequency > p->low_cut * p->min_rel_thick && realFrequency < p->high_cut;
    fftw_complex kD = get_camp(D, nzp, k);
    if (p->thickness_mode == 1) {
      /* non-constant thickness branch, src/crava.cpp:1059-1083 */
      fftw_complex kD3 = get_camp(D3, nzp, k);
      for (int l = 0; l < nt; ++l) {
        size_t o = static_cast<size_t>(k) * nt + l;
        t.wd[o] = kD;                                     /* K = DA */
        t.e1[o].re = 1.0f; t.e1[o].im = 0.0f;             /* lib_matrFillOnesVecCpx */
        t.e1[o].re /= wn[l];
        t.e2[o] = kD3;
        float errorSmoothMult = 1.0f / gn[l];
        t.e2[o].re *= errorSmoothMult;
        t.e2[o].im *= errorSmoothMult;
        /* fillInverseAbskWRobust, src/crava.cpp:1358-1384 */
        fftw_complex value = get_camp(W[l], nzp, k);
        fftw_complex valueFine = get_camp_scaled(W[l], nzp, k, 0.999f);
        float modulus = value.re * value.re + value.im * value.im;
        float modulusFine = valueFine.re * valueFine.re + valueFine.im * valueFine.im;
        float maxMod = std::max(modulus, modulusFine);
        if (maxMod > 0.0) t.e3[o] = float(1.0 / std::sqrt(maxMod));
        else t.e3[o] = wn[l] * nzp * nzp * 100.0f;
      }
      continue;
    }
    for (int l = 0; l < nt; ++l) {  /* fillkW, crava.cpp:1336-1344 */
      kW[l].re = float(get_camp(W[l], nzp, k).re);
      kW[l].im = -float(get_camp(W[l], nzp, k).im);
    }
    lib_matrProdScalVecCpx(kD, kW.data(), nt);
    for (int l = 0; l < nt; ++l) {
      size_t o = static_cast<size_t>(k) * nt + l;
      t.wd[o] = kW[l];
      /* fillkWNorm, crava.cpp:1346-1355 */
      t.e1[o].re = float(get_camp(W[l], nzp, k).re / wn[l]);
      t.e1[o].im = -float(get_camp(W[l], nzp, k).im / wn[l]);
      t.e2[o].re = float(get_camp(G[l], nzp, k).re / gn[l]);
      t.e2[o].im = -float(get_camp(G[l], nzp, k).im / gn[l]);
      t.e3[o] = 1.0f; /* lib_matrFillOnesVecCpx(errMult3) */
    }
  }
}

}  // namespace

extern "C" {

/* SeismicParametersHolder::computeCircCorrT + makeCircCorrTPosDef
 * (src/seismicparametersholder.cpp:430-499) with FFTGrid::fft1DzInPlace /
 * invFFT1DzInPlace (src/fftgrid.cpp:2002-2037): the reference's FFTW. */
int ref_circ_corr_t(const float *prior_corr_t, int n, int low_int_cut, int nzp,
                    float *circ_corr_t) {
  if (!prior_corr_t || n < 1 || prior_corr_t[0] == 0.0f) return 1;
  const int cn = nzp / 2 + 1;
  fftw_real *c = static_cast<fftw_real *>(fftw_malloc(2 * cn * sizeof(fftw_real)));
  for (int k = 0; k < 2 * cn; ++k) {
    if (k < nzp) {
      int refk = k < cn ? k : nzp - k;
      c[k] = refk < n ? prior_corr_t[refk] : 0.0f;
    } else {
      c[k] = -99999.0f;
    }
  }
  rfftwnd_plan fwd = rfftwnd_create_plan(1, &nzp, FFTW_REAL_TO_COMPLEX, FFTW_ESTIMATE | FFTW_IN_PLACE);
  rfftwnd_one_real_to_complex(fwd, c, reinterpret_cast<fftw_complex *>(c));
  fftwnd_destroy_plan(fwd);
  fftw_complex *f = reinterpret_cast<fftw_complex *>(c);
  for (int k = 0; k < cn; ++k) {
    if (k <= low_int_cut) f[k].re = 0.0;
    else f[k].re = float(std::sqrt(f[k].re * f[k].re + f[k].im * f[k].im));
    f[k].im = 0.0;
  }
  rfftwnd_plan inv = rfftwnd_create_plan(1, &nzp, FFTW_COMPLEX_TO_REAL, FFTW_ESTIMATE | FFTW_IN_PLACE);
  rfftwnd_one_complex_to_real(inv, f, c);
  fftwnd_destroy_plan(inv);
  int rc = 0;
  if (c[0] > 1.e-5f) {
    float scale = float(1.0f / c[0]);
    for (int k = 0; k < nzp; ++k) circ_corr_t[k] = c[k] * scale;
  } else {
    rc = 1;
  }
  fftw_free(c);
  return rc;
}

/* Crava::computeSyntSeismic (src/crava.cpp:1666-1719) with
 * computeSeismicImpedance (:1632-1663), constant thickness (relThick and
 * local stretch 1, the local wavelet equal to the global one): the trace
 * loop with the reference's Wavelet1D operations restated on plain arrays
 * and the reference's FFTW doing the 1-D transforms. */
int ref_synt_seismic(int nxp, int nyp, int nzp, int nx, int ny, int nz, int nt,
                     const float *A, const float *wavelet, const float *const *m,
                     float *const *out) {
  const int cnxp = nxp / 2 + 1, rnxp = 2 * cnxp, cnzp = nzp / 2 + 1, rnzp = 2 * cnzp;
  const long plane = static_cast<long>(rnxp) * nyp, rsize = plane * nzp;
  if (nz < 1 || nz > nzp || nx > nxp || ny > nyp) return 1;
  fftw_real *res = static_cast<fftw_real *>(fftw_malloc(rnzp * sizeof(fftw_real)));
  std::vector<float> imp(nzp);
  rfftwnd_plan fwd = rfftwnd_create_plan(1, &nzp, FFTW_REAL_TO_COMPLEX, FFTW_ESTIMATE | FFTW_IN_PLACE);
  rfftwnd_plan inv = rfftwnd_create_plan(1, &nzp, FFTW_COMPLEX_TO_REAL, FFTW_ESTIMATE | FFTW_IN_PLACE);
  for (int l = 0; l < nt; ++l) {
    std::vector<fftw_complex> W = spectrum1d(wavelet + static_cast<long>(l) * nzp, nzp);
    float *o = out[l];
    for (long c = 0; c < rsize; ++c) {  /* computeSeismicImpedance */
      float v = 0;
      v += m[0][c] * A[3 * l + 0];
      v += m[1][c] * A[3 * l + 1];
      v += m[2][c] * A[3 * l + 2];
      o[c] = v;
    }
    for (int i = 0; i < nx; ++i)
      for (int j = 0; j < ny; ++j) {
        const long t = i + static_cast<long>(rnxp) * j;
        int k;
        for (k = 0; k < nz; ++k) imp[k] = o[t + k * plane];
        float fac = 1.0f / static_cast<float>(nzp - nz - 1);
        for (; k < nzp; ++k) imp[k] = fac * ((k - nz) * imp[0] + (nzp - k - 1) * imp[nz - 1]);
        for (k = 0; k < nzp; ++k) res[k] = (k == nzp - 1) ? imp[0] - imp[k] : imp[k + 1] - imp[k];
        for (; k < rnzp; ++k) res[k] = 0.0f;
        rfftwnd_one_real_to_complex(fwd, res, reinterpret_cast<fftw_complex *>(res));
        fftw_complex *rc = reinterpret_cast<fftw_complex *>(res);
        for (k = 0; k < cnzp; ++k) {
          fftw_complex r = rc[k], w, sv;
          /* getCAmp(k, 1.0f): interpolation at omega = k with weight 0 */
          float omega = float(k) / 1.0f;
          int omL = int(std::floor(omega)), omU = int(std::floor(omega)) + 1;
          if (omU >= cnzp) omU -= 1;
          float dOmega = omega - float(omL);
          w.re = W[omL].re * (1.0f - dOmega) + W[omU].re * dOmega;
          w.im = (W[omL].im * (1.0f - dOmega) + W[omU].im * dOmega);
          w.re /= 1.0f; w.im /= 1.0f;
          sv.re = r.re * w.re + r.im * w.im;
          sv.im = -r.re * w.im + r.im * w.re;
          rc[k] = sv;
        }
        rfftwnd_one_complex_to_real(inv, rc, res);
        double scale = static_cast<double>(1.0 / static_cast<double>(nzp));
        for (k = 0; k < nzp; ++k) o[t + k * plane] = static_cast<fftw_real>(res[k] * scale);
      }
  }
  fftwnd_destroy_plan(fwd);
  fftwnd_destroy_plan(inv);
  fftw_free(res);
  return 0;
}

/* Crava::computeSyntSeismic (src/crava.cpp:1666-1719) with the local
 * wavelet of every trace: seisWavelet_[l]->createLocalWavelet1D(i, j)
 * (src/wavelet1D.cpp:497-505: a copy shifted and scaled by the local shift
 * and gain, Wavelet1D::shiftAndScale, src/wavelet1D.cpp:539-561) and
 * getCAmp(k, sf) with sf = relThick(i, j) * getLocalStretch(i, j) (1 for a
 * 1-D wavelet, src/wavelet.h:108) (src/wavelet.cpp:327-385).  shift / gain:
 * [ntheta][ny][nx] (ms / factor; WELLMISSING = no value) or null; rel_thick:
 * [nyp][nxp]. */
int ref_synt_seismic_local(int nxp, int nyp, int nzp, int nx, int ny, int nz, int nt,
                           const float *A, const float *wavelet, const float *const *m,
                           const double *rel_thick, float dz, const float *shift, const float *gain,
                           float *const *out) {
  const int cnxp = nxp / 2 + 1, rnxp = 2 * cnxp, cnzp = nzp / 2 + 1, rnzp = 2 * cnzp;
  const long plane = static_cast<long>(rnxp) * nyp, rsize = plane * nzp;
  if (nz < 1 || nz > nzp || nx > nxp || ny > nyp || !rel_thick) return 1;
  fftw_real *res = static_cast<fftw_real *>(fftw_malloc(rnzp * sizeof(fftw_real)));
  fftw_real *lw = static_cast<fftw_real *>(fftw_malloc(rnzp * sizeof(fftw_real)));
  fftw_complex *cw = reinterpret_cast<fftw_complex *>(lw);
  std::vector<float> imp(nzp);
  rfftwnd_plan fwd = rfftwnd_create_plan(1, &nzp, FFTW_REAL_TO_COMPLEX, FFTW_ESTIMATE | FFTW_IN_PLACE);
  rfftwnd_plan inv = rfftwnd_create_plan(1, &nzp, FFTW_COMPLEX_TO_REAL, FFTW_ESTIMATE | FFTW_IN_PLACE);
  for (int l = 0; l < nt; ++l) {
    float *o = out[l];
    for (long c = 0; c < rsize; ++c) {  /* computeSeismicImpedance */
      float v = 0;
      v += m[0][c] * A[3 * l + 0];
      v += m[1][c] * A[3 * l + 1];
      v += m[2][c] * A[3 * l + 2];
      o[c] = v;
    }
    for (int i = 0; i < nx; ++i)
      for (int j = 0; j < ny; ++j) {
        const long t = i + static_cast<long>(rnxp) * j;
        int k;
        for (k = 0; k < nz; ++k) imp[k] = o[t + k * plane];
        float fac = 1.0f / static_cast<float>(nzp - nz - 1);
        for (; k < nzp; ++k) imp[k] = fac * ((k - nz) * imp[0] + (nzp - k - 1) * imp[nz - 1]);
        for (k = 0; k < nzp; ++k) res[k] = (k == nzp - 1) ? imp[0] - imp[k] : imp[k + 1] - imp[k];
        for (; k < rnzp; ++k) res[k] = 0.0f;
        rfftwnd_one_real_to_complex(fwd, res, reinterpret_cast<fftw_complex *>(res));
        fftw_complex *rc = reinterpret_cast<fftw_complex *>(res);
        /* the local wavelet: the wavelet's spectrum, shifted and scaled */
        for (int q = 0; q < rnzp; ++q) lw[q] = q < nzp ? wavelet[static_cast<long>(l) * nzp + q] : 0.0f;
        rfftwnd_one_real_to_complex(fwd, lw, cw);
        float ts = 0.0f, g = 1.0f;
        const long so = static_cast<long>(l) * nx * ny + i + static_cast<long>(nx) * j;
        if (shift && shift[so] != -999.0f) ts = shift[so];
        if (gain && gain[so] != -999.0f) g = gain[so];
        if (shift || gain) {
          float iShift = ts / dz;
          for (k = 0; k < cnzp; k++) {
            fftw_complex am, tmp;
            am.re = float(g * cos(2.0 * (3.14159265358979323846 * (iShift) * k) / float(nzp)));
            am.im = float(g * sin(-2.0 * (3.14159265358979323846 * (iShift) * k) / float(nzp)));
            tmp.re = am.re * cw[k].re - am.im * cw[k].im;
            tmp.im = am.im * cw[k].re + am.re * cw[k].im;
            cw[k] = tmp;
          }
        }
        const float sf = static_cast<float>(rel_thick[i + static_cast<long>(nxp) * j]) * 1.0f;
        for (k = 0; k < cnzp; ++k) {
          fftw_complex r = rc[k], w, sv;  /* w = getCAmp(k, sf) */
          float omega = float(k) / sf;
          if (omega >= cnzp) { w.re = 0.0f; w.im = 0.0f; }
          else {
            int omL = int(std::floor(omega)), omU = int(std::floor(omega)) + 1;
            if (omU >= cnzp) omU -= 1;
            float dOmega = omega - float(omL);
            w.re = cw[omL].re * (1.0f - dOmega) + cw[omU].re * dOmega;
            w.im = (cw[omL].im * (1.0f - dOmega) + cw[omU].im * dOmega);
          }
          w.re /= sf; w.im /= sf;
          sv.re = r.re * w.re + r.im * w.im;
          sv.im = -r.re * w.im + r.im * w.re;
          rc[k] = sv;
        }
        rfftwnd_one_complex_to_real(inv, rc, res);
        double scale = static_cast<double>(1.0 / static_cast<double>(nzp));
        for (k = 0; k < nzp; ++k) o[t + k * plane] = static_cast<fftw_real>(res[k] * scale);
      }
  }
  fftwnd_destroy_plan(fwd);
  fftwnd_destroy_plan(inv);
  fftw_free(res);
  fftw_free(lw);
  return 0;
}

/* FFTGrid::fftInPlace, src/fftgrid.cpp:1803-1829 */
int ref_fft_r2c(float *grid, int nxp, int nyp, int nzp, int type) {
  long rsize = 2L * (nxp / 2 + 1) * nyp * nzp;
  if (type != ORC_COVARIANCE)
    multiply_by_scalar(grid, rsize, 1.0f / std::sqrt(static_cast<float>(nxp * nyp * nzp)));
  rfftwnd_plan plan = rfftw3d_create_plan(nzp, nyp, nxp, FFTW_REAL_TO_COMPLEX,
                                          FFTW_ESTIMATE | FFTW_IN_PLACE);
  rfftwnd_one_real_to_complex(plan, grid, reinterpret_cast<fftw_complex *>(grid));
  fftwnd_destroy_plan(plan);
  return 0;
}

/* FFTGrid::invFFTInPlace, src/fftgrid.cpp:1831-1862 */
int ref_fft_c2r(float *grid, int nxp, int nyp, int nzp, int type) {
  long rsize = 2L * (nxp / 2 + 1) * nyp * nzp;
  float scale;
  if (type == ORC_COVARIANCE) scale = float(1.0 / (nxp * nyp * nzp));
  else scale = float(1.0 / std::sqrt(float(nxp * nyp * nzp)));
  rfftwnd_plan plan = rfftw3d_create_plan(nzp, nyp, nxp, FFTW_COMPLEX_TO_REAL,
                                          FFTW_ESTIMATE | FFTW_IN_PLACE);
  rfftwnd_one_complex_to_real(plan, reinterpret_cast<fftw_complex *>(grid), grid);
  fftwnd_destroy_plan(plan);
  multiply_by_scalar(grid, rsize, scale);
  return 0;
}

int ref_kz_tables(const crava_oracle_params *p, float *wd, float *e1, float *e2,
                  float *e3, int *inv) {
  if (p->ntheta < 1 || p->ntheta > 16) return 1;
  KzTables t;
  build_tables(p, t);
  size_t n = t.wd.size();
  std::memcpy(wd, t.wd.data(), n * sizeof(fftw_complex));
  std::memcpy(e1, t.e1.data(), n * sizeof(fftw_complex));
  std::memcpy(e2, t.e2.data(), n * sizeof(fftw_complex));
  std::memcpy(e3, t.e3.data(), n * sizeof(float));
  std::memcpy(inv, t.inv.data(), t.inv.size() * sizeof(int));
  return 0;
}

/* Crava::computePostMeanResidAndFFTCov hot loop, src/crava.cpp:1042-1151,
 * with SeismicParametersHolder::getNextParameterCovariance
 * (src/seismicparametersholder.cpp:355-427) and
 * Crava::getNextErrorVariance (src/crava.cpp:1297-1334). */
int ref_posterior_fp32_t(const crava_oracle_params *p, const float *wd,
                         const float *e1, const float *e2, const float *e3,
                         const int *inv, float *const *mu_, float *const *data_,
                         float *const *cov_, const float *err_corr,
                         long long *chol_fail) {
  const int nxp = p->nxp, nyp = p->nyp, nzp = p->nzp, nt = p->ntheta;
  const int cnxp = nxp / 2 + 1;
  if (nt < 1 || nt > 16) return 1;
  KzTables t;
  size_t n = static_cast<size_t>(nzp) * nt;
  t.wd.assign(reinterpret_cast<const fftw_complex *>(wd), reinterpret_cast<const fftw_complex *>(wd) + n);
  t.e1.assign(reinterpret_cast<const fftw_complex *>(e1), reinterpret_cast<const fftw_complex *>(e1) + n);
  t.e2.assign(reinterpret_cast<const fftw_complex *>(e2), reinterpret_cast<const fftw_complex *>(e2) + n);
  t.e3.assign(e3, e3 + n);
  t.inv.assign(inv, inv + nzp);
  fftw_complex *mu[3], *data[16], *cov[6];
  for (int q = 0; q < 3; ++q) mu[q] = reinterpret_cast<fftw_complex *>(mu_[q]);
  for (int l = 0; l < nt; ++l) data[l] = reinterpret_cast<fftw_complex *>(data_[l]);
  for (int q = 0; q < 6; ++q) cov[q] = reinterpret_cast<fftw_complex *>(cov_[q]);
  const fftw_complex *ec = reinterpret_cast<const fftw_complex *>(err_corr);
  const double *v0 = p->var0;
  float wnc = p->wnc;

  fftw_complex *ijkData = new fftw_complex[nt], *ijkDataMean = new fftw_complex[nt];
  fftw_complex *ijkRes = new fftw_complex[nt], *ijkMean = new fftw_complex[3];
  fftw_complex *ijkAns = new fftw_complex[3];
  fftw_complex **K = alloc_mat(nt, 3), **KS = alloc_mat(nt, 3), **KScc = alloc_mat(3, nt);
  fftw_complex **parVar = alloc_mat(3, 3), **margVar = alloc_mat(nt, nt);
  fftw_complex **errVar = alloc_mat(nt, nt), **reduceVar = alloc_mat(3, 3);
  std::vector<float> A(p->A, p->A + 3 * nt);
  std::vector<float *> Arows(nt);
  for (int l = 0; l < nt; ++l) Arows[l] = &A[3 * l];
  long long fails = 0;

  for (int k = 0; k < nzp; ++k) {
    fftw_complex *kW = &t.wd[static_cast<size_t>(k) * nt];
    fftw_complex *errMult1 = &t.e1[static_cast<size_t>(k) * nt];
    fftw_complex *errMult2 = &t.e2[static_cast<size_t>(k) * nt];
    float *errMult3 = &t.e3[static_cast<size_t>(k) * nt];
    lib_matrProdDiagCpxR(kW, Arows.data(), nt, 3, K);
    bool invert_frequency = t.inv[k] != 0;
    for (int j = 0; j < nyp; ++j) {
      for (int i = 0; i < cnxp; ++i) {
        long idx = i + static_cast<long>(cnxp) * (j + static_cast<long>(nyp) * k);
        ijkMean[0] = mu[0][idx]; ijkMean[1] = mu[1][idx]; ijkMean[2] = mu[2][idx];
        for (int l = 0; l < nt; ++l) { ijkData[l] = data[l][idx]; ijkRes[l] = ijkData[l]; }

        /* getNextParameterCovariance */
        fftw_complex iiTmp = cov[0][idx], jjTmp = cov[1][idx], kkTmp = cov[2][idx];
        fftw_complex ijTmp = cov[3][idx], ikTmp = cov[4][idx], jkTmp = cov[5][idx];
        if (v0[0] != 0) iiTmp.re = iiTmp.re / static_cast<float>(v0[0]);
        if (v0[4] != 0) jjTmp.re = jjTmp.re / static_cast<float>(v0[4]);
        if (v0[8] != 0) kkTmp.re = kkTmp.re / static_cast<float>(v0[8]);
        if (v0[1] != 0) ijTmp.re = ijTmp.re / static_cast<float>(v0[1]);
        if (v0[2] != 0) ikTmp.re = ikTmp.re / static_cast<float>(v0[2]);
        if (v0[5] != 0) jkTmp.re = jkTmp.re / static_cast<float>(v0[5]);
        float ii = float(std::sqrt(iiTmp.re * iiTmp.re)), jj = float(std::sqrt(jjTmp.re * jjTmp.re));
        float kk = float(std::sqrt(kkTmp.re * kkTmp.re)), ij = float(std::sqrt(ijTmp.re * ijTmp.re));
        float ik = float(std::sqrt(ikTmp.re * ikTmp.re)), jk = float(std::sqrt(jkTmp.re * jkTmp.re));
        parVar[0][0].re = ii * static_cast<float>(v0[0]); parVar[0][0].im = 0.0;
        parVar[1][1].re = jj * static_cast<float>(v0[4]); parVar[1][1].im = 0.0;
        parVar[2][2].re = kk * static_cast<float>(v0[8]); parVar[2][2].im = 0.0;
        parVar[0][1].re = ij * static_cast<float>(v0[1]); parVar[0][1].im = 0.0;
        parVar[1][0].re = ij * static_cast<float>(v0[1]); parVar[1][0].im = -0.0f;
        parVar[0][2].re = ik * static_cast<float>(v0[2]); parVar[0][2].im = 0.0;
        parVar[2][0].re = ik * static_cast<float>(v0[2]); parVar[2][0].im = -0.0f;
        parVar[1][2].re = jk * static_cast<float>(v0[5]); parVar[1][2].im = 0.0;
        parVar[2][1].re = jk * static_cast<float>(v0[5]); parVar[2][1].im = -0.0f;

        /* getNextErrorVariance */
        fftw_complex ijkTmp = ec[idx];
        float lam = float(std::sqrt(ijkTmp.re * ijkTmp.re));
        if (invert_frequency) {
          for (int l = 0; l < nt; ++l)
            for (int m = 0; m < nt; ++m) {
              double th = p->theta_cov[l * nt + m];
              errVar[l][m].re = float(0.5 * (1.0 - wnc) * th * lam * (errMult1[l].re * errMult1[m].re + errMult1[l].im * errMult1[m].im));
              errVar[l][m].re += float(0.5 * (1.0 - wnc) * th * lam * (errMult2[l].re * errMult2[m].re + errMult2[l].im * errMult2[m].im));
              if (l == m) {
                errVar[l][m].re += float(wnc * th * errMult3[l] * errMult3[l]);
                errVar[l][m].im = 0.0;
              } else {
                errVar[l][m].im = float(0.5 * (1.0 - wnc) * th * lam * (-errMult1[l].re * errMult1[m].im + errMult1[l].im * errMult1[m].re));
                errVar[l][m].im += float(0.5 * (1.0 - wnc) * th * lam * (-errMult2[l].re * errMult2[m].im + errMult2[l].im * errMult2[m].re));
              }
            }

          lib_matrProdCpx(K, parVar, nt, 3, 3, KS);
          lib_matrProdAdjointCpx(KS, K, nt, 3, nt, margVar);
          lib_matrAddMatCpx(errVar, nt, nt, margVar);
          int cholFlag = lib_matrCholCpx(nt, margVar);
          if (cholFlag == 0) {
            lib_matrAdjoint(KS, nt, 3, KScc);
            lib_matrAXeqBMatCpx(nt, margVar, KS, 3);
            lib_matrProdCpx(KScc, KS, 3, nt, 3, reduceVar);
            lib_matrSubtMatCpx(reduceVar, 3, 3, parVar);
            lib_matrProdMatVecCpx(K, ijkMean, nt, 3, ijkDataMean);
            lib_matrSubtVecCpx(ijkDataMean, nt, ijkData);
            lib_matrProdAdjointMatVecCpx(KS, ijkData, 3, nt, ijkAns);
            lib_matrAddVecCpx(ijkAns, 3, ijkMean);
            lib_matrProdMatVecCpx(K, ijkMean, nt, 3, ijkData);
            lib_matrSubtVecCpx(ijkData, nt, ijkRes);
          } else {
            ++fails;
          }
        }
        mu[0][idx] = ijkMean[0]; mu[1][idx] = ijkMean[1]; mu[2][idx] = ijkMean[2];
        cov[0][idx] = parVar[0][0]; cov[1][idx] = parVar[1][1]; cov[2][idx] = parVar[2][2];
        cov[3][idx] = parVar[0][1]; cov[4][idx] = parVar[0][2]; cov[5][idx] = parVar[1][2];
        for (int l = 0; l < nt; ++l) data[l][idx] = ijkRes[l];
      }
    }
  }
  if (chol_fail) *chol_fail = fails;
  delete[] ijkData; delete[] ijkDataMean; delete[] ijkRes; delete[] ijkMean; delete[] ijkAns;
  free_mat(K, nt); free_mat(KS, nt); free_mat(KScc, 3); free_mat(parVar, 3);
  free_mat(margVar, nt); free_mat(errVar, nt); free_mat(reduceVar, 3);
  return 0;
}

int ref_posterior_fp32(const crava_oracle_params *p, float *const *mu,
                       float *const *data, float *const *cov,
                       const float *err_corr, long long *chol_fail) {
  if (p->ntheta < 1 || p->ntheta > 16) return 1;
  KzTables t;
  build_tables(p, t);
  return ref_posterior_fp32_t(p, reinterpret_cast<const float *>(t.wd.data()),
                              reinterpret_cast<const float *>(t.e1.data()),
                              reinterpret_cast<const float *>(t.e2.data()), t.e3.data(),
                              t.inv.data(), mu, data, cov, err_corr, chol_fail);
}

/* The timed unit (forward FFTs, solve, inverse FFTs). */
int ref_unit_fp32(const crava_oracle_params *p, float *const *mu,
                  float *const *data, float *const *cov, float *err_corr,
                  long long *chol_fail) {
  int nx = p->nxp, ny = p->nyp, nz = p->nzp;
  for (int q = 0; q < 3; ++q) ref_fft_r2c(mu[q], nx, ny, nz, ORC_PARAMETER);
  for (int l = 0; l < p->ntheta; ++l) ref_fft_r2c(data[l], nx, ny, nz, ORC_DATA);
  for (int q = 0; q < 6; ++q) ref_fft_r2c(cov[q], nx, ny, nz, ORC_COVARIANCE);
  ref_fft_r2c(err_corr, nx, ny, nz, ORC_COVARIANCE);
  int rc = ref_posterior_fp32(p, mu, data, cov, err_corr, chol_fail);
  for (int q = 0; q < 3; ++q) ref_fft_c2r(mu[q], nx, ny, nz, ORC_PARAMETER);
  for (int l = 0; l < p->ntheta; ++l) ref_fft_c2r(data[l], nx, ny, nz, ORC_DATA);
  for (int q = 0; q < 6; ++q) ref_fft_c2r(cov[q], nx, ny, nz, ORC_COVARIANCE);
  return rc;
}

unsigned int ref_rng_fill_normal(unsigned int seed, double *out, long long n) {
  RandomGen gen(seed);
  for (long long i = 0; i < n; ++i) out[i] = RandomGen::rnorm01();
  return RandomGen::seed_;
}

/* FFTGrid::fillInComplexNoise, src/fftgrid.cpp:1213-1263 */
unsigned int ref_noise_fill(float *grid, int nxp, int nyp, int nzp,
                            unsigned int seed) {
  RandomGen gen(seed);
  RandomGen *ranGen = &gen;
  fftw_complex *cvalue_ = reinterpret_cast<fftw_complex *>(grid);
  int cnxp_ = nxp / 2 + 1, nyp_ = nyp, nzp_ = nzp;
  int csize_ = cnxp_ * nyp * nzp;
  float std = float(1 / std::sqrt(2.0));
  for (int i = 0; i < csize_; i++) {
    if (((i % cnxp_) == 0) || (((i % cnxp_) == cnxp_ - 1) && ((i % 2) == 1))) {
      int xshift = i % cnxp_;
      int jkind = (i - xshift) / cnxp_;
      int jind = jkind % nyp_;
      int kind = int(jkind / nyp_);
      int jccind = jind == 0 ? 0 : nyp_ - jind;
      int kccind = kind == 0 ? 0 : nzp_ - kind;
      int jkccind = jccind + kccind * nyp_;
      if (jkccind == jkind) {
        cvalue_[i].re = float(ranGen->rnorm01());
        cvalue_[i].im = 0;
      } else if (jkccind > jkind) {
        cvalue_[i].re = float(std * ranGen->rnorm01());
        cvalue_[i].im = float(std * ranGen->rnorm01());
      } else {
        int cci = jkccind * cnxp_ + xshift;
        cvalue_[i].re = cvalue_[cci].re;
        cvalue_[i].im = -cvalue_[cci].im;
      }
    } else {
      cvalue_[i].re = float(std * ranGen->rnorm01());
      cvalue_[i].im = float(std * ranGen->rnorm01());
    }
  }
  return RandomGen::seed_;
}

/* Crava::simulate per-bin body, src/crava.cpp:1482-1521 */
int ref_sim_filter(int nxp, int nyp, int nzp, const float *const *cov_,
                   float *const *seed_, long long *chol_fail) {
  long csize = static_cast<long>(nxp / 2 + 1) * nyp * nzp;
  const fftw_complex *cv[6];
  fftw_complex *sd[3];
  for (int q = 0; q < 6; ++q) cv[q] = reinterpret_cast<const fftw_complex *>(cov_[q]);
  for (int q = 0; q < 3; ++q) sd[q] = reinterpret_cast<fftw_complex *>(seed_[q]);
  fftw_complex **ijkPostCov = alloc_mat(3, 3);
  fftw_complex ijkSeed[3];
  long long fails = 0;
  for (long i = 0; i < csize; ++i) {
    ijkPostCov[0][0] = cv[0][i]; ijkPostCov[1][1] = cv[1][i]; ijkPostCov[2][2] = cv[2][i];
    ijkPostCov[0][1] = cv[3][i]; ijkPostCov[0][2] = cv[4][i]; ijkPostCov[1][2] = cv[5][i];
    ijkPostCov[1][0].re = ijkPostCov[0][1].re; ijkPostCov[1][0].im = -ijkPostCov[0][1].im;
    ijkPostCov[2][0].re = ijkPostCov[0][2].re; ijkPostCov[2][0].im = -ijkPostCov[0][2].im;
    ijkPostCov[2][1].re = ijkPostCov[1][2].re; ijkPostCov[2][1].im = -ijkPostCov[1][2].im;
    ijkSeed[0] = sd[0][i]; ijkSeed[1] = sd[1][i]; ijkSeed[2] = sd[2][i];
    int cholFlag = lib_matrCholCpx(3, ijkPostCov);
    if (cholFlag == 0) {
      lib_matrProdCholVec(3, ijkPostCov, ijkSeed);
    } else {
      ++fails;
      for (int l = 0; l < 3; l++) { ijkSeed[l].re = 0.0; ijkSeed[l].im = 0.0; }
    }
    sd[0][i] = ijkSeed[0]; sd[1][i] = ijkSeed[1]; sd[2][i] = ijkSeed[2];
  }
  free_mat(ijkPostCov, 3);
  if (chol_fail) *chol_fail = fails;
  return 0;
}

/* State4D::merge and mergeCov (src/state4d.cpp:90-249): the reference's
 * per-bin loops with its getNextComplex order, over interleaved spectra of
 * n bins; the current covariance in the posterior's order. */
void ref_state4d_merge(long long n, const float *const *ms_, const float *const *md_,
                       const float *const *ss_, const float *const *dd_,
                       const float *const *sd_, float *const *mu_, float *const *cov_) {
  const fftw_complex *ms[3], *md[3], *ss[6], *dd[6], *sd[9];
  for (int i = 0; i < 3; ++i) {
    ms[i] = reinterpret_cast<const fftw_complex *>(ms_[i]);
    md[i] = reinterpret_cast<const fftw_complex *>(md_[i]);
  }
  for (int i = 0; i < 6; ++i) {
    ss[i] = reinterpret_cast<const fftw_complex *>(ss_[i]);
    dd[i] = reinterpret_cast<const fftw_complex *>(dd_[i]);
  }
  for (int i = 0; i < 9; ++i) sd[i] = reinterpret_cast<const fftw_complex *>(sd_[i]);
  /* sigma[0..5] = CovAlpha, CrCovAlphaBeta, CrCovAlphaRho, CovBeta,
   * CrCovBetaRho, CovRho (:150-156) */
  const int unit[6] = {0, 3, 4, 1, 5, 2};
  fftw_complex *sigma[6], *mu[3];
  for (int i = 0; i < 6; ++i) sigma[i] = reinterpret_cast<fftw_complex *>(cov_[unit[i]]);
  for (int i = 0; i < 3; ++i) mu[i] = mu_ ? reinterpret_cast<fftw_complex *>(mu_[i]) : nullptr;
  std::vector<std::vector<fftw_complex> > F(6, std::vector<fftw_complex>(6));
  std::vector<std::vector<fftw_complex> > C(3, std::vector<fftw_complex>(3));
  for (long long b = 0; b < n; ++b) {
    if (mu_) {
      fftw_complex muFullPrior[6], muCurrentPrior[3];
      for (int l = 0; l < 3; ++l) { muFullPrior[l] = ms[l][b]; muFullPrior[l + 3] = md[l][b]; }
      for (int l = 0; l < 3; l++) {
        muCurrentPrior[l].re = muFullPrior[l].re + muFullPrior[l + 3].re;
        muCurrentPrior[l].im = muFullPrior[l].im + muFullPrior[l + 3].im;
      }
      for (int l = 0; l < 3; ++l) mu[l][b] = muCurrentPrior[l];
    }
    F[0][0] = ss[0][b]; F[0][1] = ss[1][b]; F[0][2] = ss[2][b];
    F[0][3] = sd[0][b]; F[0][4] = sd[1][b]; F[0][5] = sd[2][b];
    F[1][1] = ss[3][b]; F[1][2] = ss[4][b];
    F[1][3] = sd[3][b]; F[1][4] = sd[4][b]; F[1][5] = sd[5][b];
    F[2][2] = ss[5][b];
    F[2][3] = sd[6][b]; F[2][4] = sd[7][b]; F[2][5] = sd[8][b];
    F[3][3] = dd[0][b]; F[3][4] = dd[1][b]; F[3][5] = dd[2][b];
    F[4][4] = dd[3][b]; F[4][5] = dd[4][b];
    F[5][5] = dd[5][b];
    for (int l = 0; l < 6; l++)
      for (int m = l + 1; m < 6; m++) {
        F[m][l].re = F[l][m].re;
        F[m][l].im = -F[l][m].im;
      }
    for (int l = 0; l < 3; l++)
      for (int m = 0; m < 3; m++) {
        C[l][m].re = F[l][m].re;
        C[l][m].re += F[l + 3][m + 3].re;
        C[l][m].re += F[l + 3][m].re;
        C[l][m].re += F[l][m + 3].re;
        C[l][m].im = F[l][m].im;
        C[l][m].im += F[l + 3][m + 3].im;
        C[l][m].im += F[l + 3][m].im;
        C[l][m].im += F[l][m + 3].im;
      }
    sigma[0][b] = C[0][0]; sigma[1][b] = C[0][1]; sigma[2][b] = C[0][2];
    sigma[3][b] = C[1][1]; sigma[4][b] = C[1][2]; sigma[5][b] = C[2][2];
  }
}

/* State4D::split (src/state4d.cpp:251-525): the reference's per-bin
 * sequence of lib_matr calls.  Returns the shortcut (failed Cholesky) bins. */
long long ref_state4d_split(long long n, float *const *ms_, float *const *md_,
                            float *const *ss_, float *const *dd_, float *const *sd_,
                            const float *const *mu_, const float *const *cov_) {
  fftw_complex *ms[3], *md[3], *ss[6], *dd[6], *sd[9];
  const fftw_complex *mu[3], *sigma[6];
  for (int i = 0; i < 3; ++i) {
    ms[i] = reinterpret_cast<fftw_complex *>(ms_[i]);
    md[i] = reinterpret_cast<fftw_complex *>(md_[i]);
    mu[i] = reinterpret_cast<const fftw_complex *>(mu_[i]);
  }
  for (int i = 0; i < 6; ++i) {
    ss[i] = reinterpret_cast<fftw_complex *>(ss_[i]);
    dd[i] = reinterpret_cast<fftw_complex *>(dd_[i]);
  }
  for (int i = 0; i < 9; ++i) sd[i] = reinterpret_cast<fftw_complex *>(sd_[i]);
  const int unit[6] = {0, 3, 4, 1, 5, 2};
  for (int i = 0; i < 6; ++i) sigma[i] = reinterpret_cast<const fftw_complex *>(cov_[unit[i]]);

  fftw_complex muFullPrior[6], muFullPosterior[6], muCurrentPrior[3], muCurrentPosterior[3];
  fftw_complex **sigmaFullPrior = alloc_mat(6, 6), **sigmaFullPosterior = alloc_mat(6, 6);
  fftw_complex **sigmaFullVsCurrentPrior = alloc_mat(6, 3), **adjointSandwich = alloc_mat(6, 3);
  fftw_complex **sigmaCurrentPrior = alloc_mat(3, 3), **sigmaCurrentPriorChol = alloc_mat(3, 3);
  fftw_complex **sigmaCurrentPosterior = alloc_mat(3, 3);
  fftw_complex **sandwich = alloc_mat(3, 6), **helper = alloc_mat(3, 6);
  long long counter = 0;
  for (long long b = 0; b < n; ++b) {
    for (int l = 0; l < 3; ++l) { muFullPrior[l] = ms[l][b]; muFullPrior[l + 3] = md[l][b]; }
    fftw_complex **F = sigmaFullPrior;
    F[0][0] = ss[0][b]; F[0][1] = ss[1][b]; F[0][2] = ss[2][b];
    F[0][3] = sd[0][b]; F[0][4] = sd[1][b]; F[0][5] = sd[2][b];
    F[1][1] = ss[3][b]; F[1][2] = ss[4][b];
    F[1][3] = sd[3][b]; F[1][4] = sd[4][b]; F[1][5] = sd[5][b];
    F[2][2] = ss[5][b];
    F[2][3] = sd[6][b]; F[2][4] = sd[7][b]; F[2][5] = sd[8][b];
    F[3][3] = dd[0][b]; F[3][4] = dd[1][b]; F[3][5] = dd[2][b];
    F[4][4] = dd[3][b]; F[4][5] = dd[4][b];
    F[5][5] = dd[5][b];
    for (int l = 0; l < 3; ++l) muCurrentPosterior[l] = mu[l][b];
    sigmaCurrentPosterior[0][0] = sigma[0][b]; sigmaCurrentPosterior[0][1] = sigma[1][b];
    sigmaCurrentPosterior[0][2] = sigma[2][b]; sigmaCurrentPosterior[1][1] = sigma[3][b];
    sigmaCurrentPosterior[1][2] = sigma[4][b]; sigmaCurrentPosterior[2][2] = sigma[5][b];
    sigmaCurrentPosterior[1][0] = sigmaCurrentPosterior[0][1];
    sigmaCurrentPosterior[2][0] = sigmaCurrentPosterior[0][2];
    sigmaCurrentPosterior[2][1] = sigmaCurrentPosterior[1][2];
    for (int l = 0; l < 6; l++)
      for (int m = l + 1; m < 6; m++) {
        F[m][l].re = F[l][m].re;
        F[m][l].im = -F[l][m].im;
      }
    for (int l = 0; l < 3; l++) {
      muCurrentPrior[l].re = muFullPrior[l].re + muFullPrior[l + 3].re;
      muCurrentPrior[l].im = muFullPrior[l].im + muFullPrior[l + 3].im;
    }
    for (int l = 0; l < 6; l++)
      for (int m = 0; m < 3; m++) {
        sigmaFullVsCurrentPrior[l][m].re = F[l][m].re + F[l][m + 3].re;
        sigmaFullVsCurrentPrior[l][m].im = F[l][m].im + F[l][m + 3].im;
      }
    for (int l = 0; l < 3; l++)
      for (int m = 0; m < 3; m++) {
        sigmaCurrentPrior[l][m].re = sigmaFullVsCurrentPrior[l][m].re + sigmaFullVsCurrentPrior[l + 3][m].re;
        sigmaCurrentPrior[l][m].im = sigmaFullVsCurrentPrior[l][m].im + sigmaFullVsCurrentPrior[l + 3][m].im;
      }
    lib_matrCopyCpx(sigmaCurrentPrior, 3, 3, sigmaCurrentPriorChol);
    lib_matrAdjoint(sigmaFullVsCurrentPrior, 6, 3, sandwich);
    int flag = lib_matrCholCpx(3, sigmaCurrentPriorChol);
    if (flag == 0) {
      lib_matrAXeqBMatCpx(3, sigmaCurrentPriorChol, sandwich, 6);
      lib_matrSubtMatCpx(sigmaCurrentPrior, 3, 3, sigmaCurrentPosterior);
      lib_matrProdCpx(sigmaCurrentPosterior, sandwich, 3, 3, 6, helper);
      lib_matrAdjoint(sandwich, 3, 6, adjointSandwich);
      lib_matrProdCpx(adjointSandwich, helper, 6, 3, 6, sigmaFullPosterior);
      lib_matrAddMatCpx(sigmaFullPrior, 6, 6, sigmaFullPosterior);
      lib_matrSubtVecCpx(muCurrentPrior, 3, muCurrentPosterior);
      lib_matrProdMatVecCpx(adjointSandwich, muCurrentPosterior, 6, 3, muFullPosterior);
      lib_matrAddVecCpx(muFullPrior, 6, muFullPosterior);
    } else {
      counter++;
      lib_matrCopyCpx(sigmaFullPrior, 6, 6, sigmaFullPosterior);
      for (int l = 0; l < 6; l++) muFullPosterior[l] = muFullPrior[l];
    }
    fftw_complex **P = sigmaFullPosterior;
    ss[0][b] = P[0][0]; ss[1][b] = P[0][1]; ss[2][b] = P[0][2];
    sd[0][b] = P[0][3]; sd[1][b] = P[0][4]; sd[2][b] = P[0][5];
    ss[3][b] = P[1][1]; ss[4][b] = P[1][2];
    sd[3][b] = P[1][3]; sd[4][b] = P[1][4]; sd[5][b] = P[1][5];
    ss[5][b] = P[2][2];
    sd[6][b] = P[2][3]; sd[7][b] = P[2][4]; sd[8][b] = P[2][5];
    dd[0][b] = P[3][3]; dd[1][b] = P[3][4]; dd[2][b] = P[3][5];
    dd[3][b] = P[4][4]; dd[4][b] = P[4][5];
    dd[5][b] = P[5][5];
    for (int l = 0; l < 3; ++l) { ms[l][b] = muFullPosterior[l]; md[l][b] = muFullPosterior[l + 3]; }
  }
  free_mat(sigmaFullPrior, 6); free_mat(sigmaFullPosterior, 6);
  free_mat(sigmaFullVsCurrentPrior, 6); free_mat(adjointSandwich, 6);
  free_mat(sigmaCurrentPrior, 3); free_mat(sigmaCurrentPriorChol, 3);
  free_mat(sigmaCurrentPosterior, 3); free_mat(sandwich, 3); free_mat(helper, 3);
  return counter;
}

/* Crava::divideDataByScaleWavelet (src/crava.cpp:591-722) with
 * computeAdjustmentFactor (:725-817), 1-D wavelets, without the closing
 * interpolateSeismic, on the reference's FFTW: every transform the
 * reference makes per trace (the global wavelet back to the time domain by
 * the local copy's constructor and forward again by computeAdjustmentFactor,
 * the local wavelet's shiftAndScale, inverse, difference wavelets and
 * forward transforms, the reflection-coefficient covariance, the data
 * trace) is made here with rfftwnd in the same order. */
int ref_divide_data(const crava_oracle_params *p, float *const *data, const float *cov_col,
                    const double *rel_thick, int nx, int ny, float dz, const float *shift,
                    const float *gain) {
  const int nxp = p->nxp, nyp = p->nyp, nzp = p->nzp, nt = p->ntheta, nz = p->nz;
  const int cnzp = nzp / 2 + 1, rnzp = 2 * cnzp, rnxp = 2 * (nxp / 2 + 1);
  const float RM = -99999.0f, tolFac = 0.05f;
  rfftwnd_plan fwd = rfftwnd_create_plan(1, &nzp, FFTW_REAL_TO_COMPLEX, FFTW_ESTIMATE | FFTW_IN_PLACE);
  rfftwnd_plan inv = rfftwnd_create_plan(1, &nzp, FFTW_COMPLEX_TO_REAL, FFTW_ESTIMATE | FFTW_IN_PLACE);
  fftw_real *gw = static_cast<fftw_real *>(fftw_malloc(rnzp * sizeof(fftw_real)));  /* global wavelet */
  fftw_real *lw = static_cast<fftw_real *>(fftw_malloc(rnzp * sizeof(fftw_real)));  /* local wavelet */
  fftw_real *e1 = static_cast<fftw_real *>(fftw_malloc(rnzp * sizeof(fftw_real)));
  fftw_real *e2 = static_cast<fftw_real *>(fftw_malloc(rnzp * sizeof(fftw_real)));
  fftw_real *e3 = static_cast<fftw_real *>(fftw_malloc(rnzp * sizeof(fftw_real)));
  fftw_real *rc = static_cast<fftw_real *>(fftw_malloc(rnzp * sizeof(fftw_real)));
  fftw_real *rd = static_cast<fftw_real *>(fftw_malloc(rnzp * sizeof(fftw_real)));
  std::vector<fftw_complex> adj(cnzp);
  auto to_c = [](fftw_real *r) { return reinterpret_cast<fftw_complex *>(r); };
  /* Wavelet::invFFT1DInPlace (src/wavelet.cpp:264-280) */
  auto inverse = [&](fftw_real *r) {
    rfftwnd_one_complex_to_real(inv, to_c(r), r);
    double scale = static_cast<double>(1.0 / static_cast<double>(nzp));
    for (int i = 0; i < nzp; i++) r[i] = static_cast<fftw_real>(r[i] * scale);
  };
  auto forward = [&](fftw_real *r) { rfftwnd_one_real_to_complex(fwd, r, to_c(r)); };
  /* Wavelet::getCAmp(k, scale), k < cnzp (src/wavelet.cpp:327-385) */
  auto camp = [&](const fftw_complex *c, int k, float scale) {
    fftw_complex value;
    float omega = float(k) / scale;
    if (omega >= cnzp) { value.re = 0.0f; value.im = 0.0f; }
    else {
      int omL = int(std::floor(omega)), omU = int(std::floor(omega)) + 1;
      if (omU >= cnzp) omU -= 1;
      float dOmega = omega - float(omL);
      value.re = c[omL].re * (1.0f - dOmega) + c[omU].re * dOmega;
      value.im = (c[omL].im * (1.0f - dOmega) + c[omU].im * dOmega);
    }
    value.re /= scale; value.im /= scale;
    return value;
  };
  auto band_norm = [&](const fftw_complex *c) {  /* findNormWithinFrequencyBand */
    double norm2 = 0.0;
    float dOmega = 1.0 / (nzp * dz * 0.001);
    int loI = std::max<int>(0, static_cast<int>(std::floor(p->low_cut / dOmega)));
    int hiI = std::min<int>(cnzp, static_cast<int>(std::ceil(p->high_cut / dOmega)));
    double fac = 1.0 / double(nzp);
    for (int i = loI; i < hiI; i++) norm2 += static_cast<double>(2.0 * fac * (c[i].re * c[i].re + c[i].im * c[i].im));
    if (loI == 0) norm2 -= fac * (c[0].re * c[0].re + c[0].im * c[0].im);
    return static_cast<float>(std::sqrt(norm2));
  };
  const float sq = static_cast<float>(std::sqrt(static_cast<float>(nzp)));
  for (int l = 0; l < nt; ++l) {
    for (int i = 0; i < rnzp; ++i) gw[i] = i < nzp ? p->wavelet[static_cast<long>(l) * nzp + i] : 0.0f;
    bool gReal = true;
    const float wn = p->wavelet_norm ? p->wavelet_norm[l] : [&] {
      double s = 0.0;
      for (int i = 0; i < nzp; i++) s += static_cast<double>(gw[i] * gw[i]);
      return static_cast<float>(std::sqrt(s));
    }();
    const float errorVar = static_cast<float>(p->theta_cov[l * nt + l]);
    for (int i = 0; i < nxp; i++)
      for (int j = 0; j < nyp; j++) {
        int iInd = i, jInd = j;
        if (iInd > 3 * nx - 1) iInd = 0;
        if (jInd > 3 * ny - 1) jInd = 0;
        if ((iInd > (nxp + nx) / 2)) iInd = nxp - iInd;
        if (iInd >= nx) iInd = 2 * nx - iInd - 1;
        if (jInd > (nyp + ny) / 2) jInd = nyp - jInd;
        if (jInd >= ny) jInd = 2 * ny - jInd - 1;
        /* the data trace */
        const long t0 = i + static_cast<long>(rnxp) * j, plane = static_cast<long>(rnxp) * nyp;
        for (int k = 0; k < nzp; k++) {
          rd[k] = data[l][t0 + k * plane] / sq;
          if (k > nz) {
            float dist;
            {
              float taper = static_cast<float>((std::min(nz, nzp - nz) / 2.1));
              int below = nzp - k, above = k - (nz - 1);
              dist = above < below ? static_cast<float>(above / taper) : static_cast<float>(below / taper);
            }
            rd[k] *= std::max<float>(1 - dist * dist, 0);
          }
        }
        forward(rd);
        /* createLocalWavelet1D: the copy constructor returns the global
         * wavelet to the time domain, then shiftAndScale */
        if (!gReal) { inverse(gw); gReal = true; }
        for (int q = 0; q < rnzp; ++q) lw[q] = q < nzp ? gw[q] : 0.0f;
        float ts = 0.0f, g = 1.0f;
        if (iInd >= 0 && iInd < nx && jInd >= 0 && jInd < ny) {  /* src/wavelet.cpp:1143-1172 */
          const long o = static_cast<long>(l) * nx * ny + iInd + static_cast<long>(nx) * jInd;
          if (shift && shift[o] != -999.0f) ts = shift[o];
          if (gain && gain[o] != -999.0f) g = gain[o];
        }
        forward(lw);
        {
          float iShift = ts / dz;
          fftw_complex *c = to_c(lw);
          for (int k = 0; k < cnzp; k++) {
            fftw_complex am, tmp;
            am.re = float(g * cos(2.0 * (3.14159265358979323846 * (iShift) * k) / float(nzp)));
            am.im = float(g * sin(-2.0 * (3.14159265358979323846 * (iShift) * k) / float(nzp)));
            tmp.re = am.re * c[k].re - am.im * c[k].im;
            tmp.im = am.im * c[k].re + am.re * c[k].im;
            c[k] = tmp;
          }
        }
        double relT = rel_thick[i + static_cast<long>(nxp) * j];
        double sfLoc = relT * 1.0f;
        /* computeAdjustmentFactor: the reflection-coefficient covariance */
        {
          double eiVar = 0.0;
          for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++)
              eiVar += p->A[3 * l + a] * static_cast<float>(p->var0[3 * a + b]) * p->A[3 * l + b];
          float constant = cov_col[0];
          for (int k = 0; k < nzp; k++) {
            int refk = k < nzp / 2 + 1 ? k : nzp - k;
            float corr = refk < nz ? cov_col[refk] / constant : 0.0f;
            rc[k] = static_cast<fftw_real>(eiVar * corr);
          }
          fftw_real first = rc[0], prev = rc[nzp - 1];
          for (int k = 0; k < nzp - 1; k++) {
            fftw_real curr = rc[k], next = rc[k + 1];
            rc[k] = 2 * curr - next - prev;
            prev = curr;
          }
          rc[nzp - 1] = 2 * rc[nzp - 1] - first - prev;
          forward(rc);
        }
        /* difference wavelets of the local wavelet (back in time first) */
        inverse(lw);
        for (int k = 0; k < rnzp; k++) e1[k] = k < nzp ? ((k == nzp - 1) ? lw[0] - lw[k] : lw[k + 1] - lw[k]) : RM;
        for (int k = 0; k < rnzp; k++) e2[k] = k < nzp ? ((k == 0) ? e1[0] - e1[nzp - 1] : e1[k] - e1[k - 1]) : RM;
        for (int k = 0; k < rnzp; k++) {
          if (k >= nzp) { e3[k] = RM; continue; }
          if (k == 0) e3[k] = static_cast<fftw_real>(0.5 * (e2[k + 1] - e2[nzp - 1]));
          else if (k == nzp - 1) e3[k] = static_cast<fftw_real>(0.5 * (e2[0] - e2[k - 1]));
          else e3[k] = static_cast<fftw_real>(0.5 * (e2[k + 1] - e2[k - 1]));
        }
        forward(e3);
        {
          float c3 = 1.0f / band_norm(to_c(e3));
          for (int k = 0; k < rnzp; k++) e3[k] = k < nzp ? e3[k] * c3 : RM;
        }
        forward(lw);
        if (gReal) { forward(gw); gReal = false; }  /* wGlobal->fft1DInPlace() */
        float modW = wn;
        modW *= modW;
        float maxfrequency = static_cast<float>((nzp / 2) * 1000.0 * nz) / static_cast<float>(p->lz * nzp);
        modW *= maxfrequency / static_cast<float>(p->high_cut);
        const fftw_complex *W = to_c(gw), *Wl = to_c(lw), *E3 = to_c(e3), *R = to_c(rc);
        float sf = static_cast<float>(sfLoc);
        for (int k = 0; k < cnzp; k++) {
          fftw_complex wLoc = camp(Wl, k, sf);
          float wLoc2 = (wLoc.re * wLoc.re + wLoc.im * wLoc.im);
          fftw_complex wGlob = W[k];
          float wGlob2 = (wGlob.re * wGlob.re + wGlob.im * wGlob.im);
          fftw_complex eSkLoc = camp(Wl, k, sf);
          float sizeESkLoc = (eSkLoc.re * eSkLoc.re + eSkLoc.im * eSkLoc.im) / (wn * wn);
          eSkLoc = camp(E3, k, sf);
          sizeESkLoc += eSkLoc.re * eSkLoc.re + eSkLoc.im * eSkLoc.im;
          fftw_complex eSkGlob = Wl[k];
          float sizeESkGlob = (eSkGlob.re * eSkGlob.re + eSkGlob.im * eSkGlob.im) / (wn * wn);
          eSkGlob = E3[k];
          sizeESkGlob += eSkGlob.re * eSkGlob.re + eSkGlob.im * eSkGlob.im;
          float sigma2Loc = errorVar * (p->wnc + (1.0f - p->wnc) * 0.5f * sizeESkLoc);
          float sigma2Glob = errorVar * (p->wnc + (1.0f - p->wnc) * 0.5f * sizeESkGlob);
          float tau2 = std::fabs(static_cast<float>(R[k].re));
          float wGlob2Adj = wGlob2, wLoc2Adj = wLoc2;
          if (wGlob2 < tolFac * modW) wGlob2Adj = float(0.5f * (wGlob2 + tolFac * modW));
          if (wLoc2 < tolFac * modW) wLoc2Adj = float(0.5f * (wLoc2 + tolFac * modW));
          if (wLoc2Adj < tolFac * wGlob2Adj) {
            wLoc2Adj = float(0.5f * (wLoc2 + tolFac * wGlob2Adj));
            sigma2Loc *= wLoc2Adj / wLoc2;
          }
          adj[k].re = (wLoc.re / (tau2 * wLoc2Adj + sigma2Loc)) / (wGlob2Adj / (tau2 * wGlob2 + sigma2Glob));
          adj[k].im = (wLoc.im / (tau2 * wLoc2Adj + sigma2Loc)) / (wGlob2Adj / (tau2 * wGlob2 + sigma2Glob));
        }
        double deltaF = static_cast<double>(nz) * 1000.0 / (relT * p->lz * static_cast<double>(nzp));
        fftw_complex *cd = to_c(rd);
        for (int k = 0; k < cnzp; k++) {
          if ((deltaF * k < p->high_cut) && (deltaF * k > p->low_cut)) {
            fftw_real tmp = cd[k].re * adj[k].re - cd[k].im * adj[k].im;
            cd[k].im = cd[k].im * adj[k].re + cd[k].re * adj[k].im;
            cd[k].re = tmp;
          } else {
            cd[k].im = 0.0f;
            cd[k].re = 0.0f;
          }
        }
        rfftwnd_one_complex_to_real(inv, cd, rd);
        for (int k = 0; k < nzp; k++) data[l][t0 + k * plane] = rd[k] / sq;
      }
  }
  fftw_free(gw); fftw_free(lw); fftw_free(e1); fftw_free(e2); fftw_free(e3); fftw_free(rc); fftw_free(rd);
  fftwnd_destroy_plan(fwd);
  fftwnd_destroy_plan(inv);
  return 0;
}

/* Crava::multiplyDataByScaleWaveletAndWriteToFile (src/crava.cpp:819-885)
 * before the file write, on time-domain residual grids, with the
 * reference's FFTW per trace and the local wavelet made as
 * createLocalWavelet1D makes it (copy, forward transform, shiftAndScale). */
int ref_multiply_data(const crava_oracle_params *p, float *const *data, const double *rel_thick,
                      int nx, int ny, float dz, const float *shift, const float *gain) {
  const int nxp = p->nxp, nyp = p->nyp, nzp = p->nzp, nt = p->ntheta;
  const int cnzp = nzp / 2 + 1, rnzp = 2 * cnzp, rnxp = 2 * (nxp / 2 + 1);
  rfftwnd_plan fwd = rfftwnd_create_plan(1, &nzp, FFTW_REAL_TO_COMPLEX, FFTW_ESTIMATE | FFTW_IN_PLACE);
  rfftwnd_plan inv = rfftwnd_create_plan(1, &nzp, FFTW_COMPLEX_TO_REAL, FFTW_ESTIMATE | FFTW_IN_PLACE);
  fftw_real *rd = static_cast<fftw_real *>(fftw_malloc(rnzp * sizeof(fftw_real)));
  fftw_real *lw = static_cast<fftw_real *>(fftw_malloc(rnzp * sizeof(fftw_real)));
  fftw_complex *cd = reinterpret_cast<fftw_complex *>(rd), *cw = reinterpret_cast<fftw_complex *>(lw);
  for (int l = 0; l < nt; l++) {
    const long plane = static_cast<long>(rnxp) * nyp;
    for (int i = 0; i < nx; i++)
      for (int j = 0; j < ny; j++) {
        float sf = static_cast<float>(rel_thick[i + static_cast<long>(nxp) * j]) * 1.0f;
        const long t0 = i + static_cast<long>(rnxp) * j;
        for (int k = 0; k < nzp; k++)
          rd[k] = data[l][t0 + k * plane] / static_cast<float>(std::sqrt(static_cast<float>(nzp)));
        rfftwnd_one_real_to_complex(fwd, rd, cd);
        for (int q = 0; q < rnzp; ++q) lw[q] = q < nzp ? p->wavelet[static_cast<long>(l) * nzp + q] : 0.0f;
        rfftwnd_one_real_to_complex(fwd, lw, cw);
        float ts = 0.0f, g = 1.0f;
        const long o = static_cast<long>(l) * nx * ny + i + static_cast<long>(nx) * j;
        if (shift && shift[o] != -999.0f) ts = shift[o];
        if (gain && gain[o] != -999.0f) g = gain[o];
        float iShift = ts / dz;
        for (int k = 0; k < cnzp; k++) {
          fftw_complex am, tmp;
          am.re = float(g * cos(2.0 * (3.14159265358979323846 * (iShift) * k) / float(nzp)));
          am.im = float(g * sin(-2.0 * (3.14159265358979323846 * (iShift) * k) / float(nzp)));
          tmp.re = am.re * cw[k].re - am.im * cw[k].im;
          tmp.im = am.im * cw[k].re + am.re * cw[k].im;
          cw[k] = tmp;
        }
        for (int k = 0; k < cnzp; k++) {
          fftw_complex sv;  /* getCAmp(k, sf), k < cnzp */
          float omega = float(k) / sf;
          if (omega >= cnzp) { sv.re = 0.0f; sv.im = 0.0f; }
          else {
            int omL = int(std::floor(omega)), omU = int(std::floor(omega)) + 1;
            if (omU >= cnzp) omU -= 1;
            float dOmega = omega - float(omL);
            sv.re = cw[omL].re * (1.0f - dOmega) + cw[omU].re * dOmega;
            sv.im = (cw[omL].im * (1.0f - dOmega) + cw[omU].im * dOmega);
          }
          sv.re /= sf; sv.im /= sf;
          fftw_real tmp = cd[k].re * sv.re + cd[k].im * sv.im;
          cd[k].im = cd[k].im * sv.re - cd[k].re * sv.im;
          cd[k].re = tmp;
        }
        rfftwnd_one_complex_to_real(inv, cd, rd);
        for (int k = 0; k < nzp; k++)
          data[l][t0 + k * plane] = rd[k] / static_cast<float>(std::sqrt(static_cast<double>(nzp)));
      }
  }
  fftw_free(rd); fftw_free(lw);
  fftwnd_destroy_plan(fwd);
  fftwnd_destroy_plan(inv);
  return 0;
}

}  /* extern "C" */
