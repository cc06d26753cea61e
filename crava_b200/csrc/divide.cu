// divide.cu -- the data divided by the local scale wavelet (non-constant
// thickness), on the device.
//
// Replaces Crava::divideDataByScaleWavelet (src/crava.cpp:591-722) with
// Crava::computeAdjustmentFactor (:725-817) for one-dimensional wavelets,
// up to (not including) its final FFTGrid::interpolateSeismic of
// low-energy traces.  Per trace (i, j) of each angle the reference
// transforms the tapered trace along z, multiplies every in-band bin by an
// adjustment factor built from the trace's stretched local wavelet, zeroes
// the others and transforms back.
//
// B200 form.  Two neighbouring traces of the padded real layout are one
// complex line of its complex view, so one batched complex z pass of the
// grid transforms all traces in pairs (z = a + i b); the filter kernel
// separates each pair's spectra at bins k and nzp - k, multiplies each by
// its own factor, recombines them and the inverse z pass returns both
// traces.  The factor of a trace depends on it only through its relative
// thickness (the stretch of getCAmp(k, scale)) and, with local shift and
// gain grids, a phase ramp and a gain: it is evaluated on the fly from
// per-angle tables (wavelet spectrum, normalised third-difference
// spectrum, reflection-coefficient spectrum) built once per call by
// k_div_tables, instead of the reference's three wavelet transforms and
// one covariance transform per trace.
#include <math.h>

#include <cstring>
#include <vector>

#include "context.cuh"
#include "fft_core.cuh"

using namespace crava;

namespace {

constexpr int kThreads = 256;
constexpr int kTabThreads = 256;
constexpr float kMissing = -99999.0f;  // RMISSING, src/definitions.h:35

// Per-angle scalars of computeAdjustmentFactor.
struct DivScalars {
  float wn2;        // wLocal->getNorm()^2 (the global wavelet's norm)
  float modW;       // tolFac scale: |w|^2 (nzp/2 maxfrequency) / highCut
  float error_var;  // errThetaCov_[l][l]
  float e3_inv;     // 1 / normF3, the band norm of the third difference
};

struct DivTables {
  float2 *W;         // [nt][cnzp] wavelet spectrum (Wavelet::fft1DInPlace)
  float2 *E3;        // [nt][cnzp] third-difference spectrum (unnormalised)
  float *tau2;       // [nt][cnzp] |Re FFT(reflection-coefficient time covariance)|
  DivScalars *sc;    // [nt]
};

// ------------------------------------------------------------------ tables
// Follows computeAdjustmentFactor's preparation (src/crava.cpp:736-777):
// the reflection-coefficient time covariance
// (computeReflectionCoefficientTimeCovariance, :476-508, on
// getPriorCorrTFiltered, src/seismicparametersholder.cpp:504-530), the
// difference wavelets (src/wavelet1D.cpp:420-479), the band norm
// (Wavelet::findNormWithinFrequencyBand, src/wavelet.cpp:811-833) and the
// wavelet's norm scale modW.  Unnormalised forward DFTs in double, rounded
// to float, stand in for FFTW's single-precision transforms.
struct DivConsts {
  const float *wav;      // [nt][nzp]
  const float *wnorm;    // [nt] or null (time-domain norm)
  const float *A;        // [nt][3]
  const double *var0;    // [3][3]
  const double *theta;   // [nt][nt]
  const float *cov_alpha;  // real-domain covAlpha grid; column (0, 0, k)
  long long col_stride;    // rnxp nyp
  int nzp, nt, nz;
  double lz;
  float dz, low_cut, high_cut;
};

// Spectra: grid (angle, chunk of kTabThreads bins); each block forms the
// angle's time-domain sequences in shared memory, each thread one bin.
__global__ void __launch_bounds__(kTabThreads) k_div_spectra(const __grid_constant__ DivConsts q, DivTables t) {
  extern __shared__ double shd[];
  const int l = blockIdx.x, tid = threadIdx.x, nth = blockDim.x;
  const int nzp = q.nzp, cnzp = nzp / 2 + 1;
  double *cs = shd;
  double *sn = cs + nzp;
  float *w = reinterpret_cast<float *>(sn + nzp);
  float *e = w + nzp, *f = e + nzp, *g = f + nzp, *r = g + nzp;
  const float *wl = q.wav + (long long)l * nzp;
  for (int m = tid; m < nzp; m += nth) {
    double sv, cv;
    sincospi(2.0 * m / nzp, &sv, &cv);
    cs[m] = cv; sn[m] = sv;
    w[m] = wl[m];
  }
  // reflection-coefficient time covariance: eiVar corrT, then the cyclic
  // second difference 2 c[i] - c[i+1] - c[i-1] in float
  double eiVar = 0.0;
  for (int p = 0; p < 3; ++p)
    for (int k = 0; k < 3; ++k)
      eiVar += (double)__fmul_rn(__fmul_rn(q.A[3 * l + p], (float)q.var0[3 * p + k]), q.A[3 * l + k]);
  // (no covariance grid: the wavelet spectrum alone is wanted)
  const float constant = q.cov_alpha ? q.cov_alpha[0] : 1.0f;
  for (int i = tid; i < nzp; i += nth) {
    const int refk = i < nzp / 2 + 1 ? i : nzp - i;
    const float corr = (q.cov_alpha && refk < q.nz) ? __fdiv_rn(q.cov_alpha[refk * q.col_stride], constant) : 0.0f;
    e[i] = (float)(eiVar * (double)corr);
  }
  __syncthreads();
  for (int i = tid; i < nzp; i += nth) {
    const float curr = e[i], next = e[(i + 1) % nzp], prev = e[(i + nzp - 1) % nzp];
    r[i] = __fsub_rn(__fsub_rn(__fmul_rn(2.0f, curr), next), prev);
  }
  __syncthreads();
  // difference wavelets: forward, backward, central (cyclic)
  for (int i = tid; i < nzp; i += nth) e[i] = (i == nzp - 1) ? w[0] - w[i] : w[i + 1] - w[i];
  __syncthreads();
  for (int i = tid; i < nzp; i += nth) f[i] = (i == 0) ? e[0] - e[nzp - 1] : e[i] - e[i - 1];
  __syncthreads();
  for (int i = tid; i < nzp; i += nth) {
    const float d = (i == 0) ? f[1] - f[nzp - 1] : (i == nzp - 1) ? f[0] - f[i - 1] : f[i + 1] - f[i - 1];
    g[i] = (float)(0.5 * (double)d);
  }
  __syncthreads();
  const int k = blockIdx.y * nth + tid;
  if (k >= cnzp) return;
  double wr = 0, wi = 0, gr = 0, gi = 0, rr = 0;
  int m = 0;  // k n mod nzp, stepped
  for (int n = 0; n < nzp; ++n) {
    const double c = cs[m], sv = -sn[m];
    wr += w[n] * c; wi += w[n] * sv;
    gr += g[n] * c; gi += g[n] * sv;
    rr += r[n] * c;
    m += k;
    if (m >= nzp) m -= nzp;
  }
  const long long o = (long long)l * cnzp + k;
  t.W[o] = make_float2((float)wr, (float)wi);
  t.E3[o] = make_float2((float)gr, (float)gi);
  t.tau2[o] = fabsf((float)rr);
}

// Scalars: one block per angle (band norm of the third difference, the
// wavelet's norm, modW, the noise variance).
__global__ void __launch_bounds__(kTabThreads) k_div_scalars(const __grid_constant__ DivConsts q, DivTables t) {
  __shared__ double red[2 * kTabThreads];
  const int l = blockIdx.x, tid = threadIdx.x, nth = blockDim.x;
  const int nzp = q.nzp, cnzp = nzp / 2 + 1;
  const float *wl = q.wav + (long long)l * nzp;
  const float2 *El = t.E3 + (long long)l * cnzp;
  const float dOmega = (float)(1.0 / ((double)__fmul_rn((float)nzp, q.dz) * 0.001));
  const int loI = max(0, (int)floorf(__fdiv_rn(q.low_cut, dOmega)));
  const int hiI = min(cnzp, (int)ceilf(__fdiv_rn(q.high_cut, dOmega)));
  const double fac = 1.0 / (double)nzp;
  double sw = 0.0, nb = 0.0;
  for (int i = tid; i < nzp; i += nth) sw += (double)(wl[i] * wl[i]);
  for (int i = loI + tid; i < hiI; i += nth) {
    const float2 v = El[i];
    nb += 2.0 * fac * (double)__fadd_rn(__fmul_rn(v.x, v.x), __fmul_rn(v.y, v.y));
  }
  red[tid] = sw; red[nth + tid] = nb;
  __syncthreads();
  for (int off = nth / 2; off > 0; off >>= 1) {
    if (tid < off) { red[tid] += red[tid + off]; red[nth + tid] += red[nth + tid + off]; }
    __syncthreads();
  }
  if (tid != 0) return;
  double norm2 = red[nth];
  if (loI == 0) {
    const float2 v = El[0];
    norm2 -= fac * (double)__fadd_rn(__fmul_rn(v.x, v.x), __fmul_rn(v.y, v.y));
  }
  const float wn = q.wnorm ? q.wnorm[l] : (float)sqrt(red[0]);
  const float maxfrequency = __fdiv_rn((float)((double)(nzp / 2) * 1000.0 * (double)q.nz),
                                       (float)(q.lz * (double)nzp));
  DivScalars sc;
  sc.wn2 = __fmul_rn(wn, wn);
  sc.modW = __fmul_rn(sc.wn2, __fdiv_rn(maxfrequency, q.high_cut));
  sc.error_var = (float)q.theta[(long long)l * q.nt + l];
  sc.e3_inv = __fdiv_rn(1.0f, (float)sqrt(norm2));  // multiplyRAmpByConstant(1/normF3)
  t.sc[l] = sc;
}

// ------------------------------------------------------------ pre / post
struct DivPassArgs {
  float *grid;
  float *pads;  // (rnxp - nxp) floats per row
  int nxp, nyp, nzp, rnxp, nz;
  float sq;     // float(sqrt(float(nzp)))
};

// FFTGrid::getDistToBoundary (src/fftgrid.cpp:1374-1414) for i < np.
__device__ __forceinline__ float dist_to_boundary(int i, int n, int np) {
  if (i < n) return 0.0f;
  const float taper = (float)((double)min(n, np - n) / 2.1);
  const int below = np - i, above = i - (n - 1);
  return above < below ? __fdiv_rn((float)above, taper) : __fdiv_rn((float)below, taper);
}

// Before the forward pass: value / sqrt(nzp), tapered below the volume
// (src/crava.cpp:647-655); the row padding is set aside.  One warp per
// row of the padded layout, float2 (two traces) per lane.
constexpr int kRowsPerBlock = kThreads / 32;

__global__ void __launch_bounds__(kThreads) k_div_pre(const __grid_constant__ DivPassArgs a) {
  const int row = blockIdx.x * kRowsPerBlock + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (row >= a.nyp * a.nzp) return;
  const int k = row / a.nyp, cnxp = a.rnxp / 2;
  float2 *__restrict__ r = reinterpret_cast<float2 *>(a.grid + (long long)row * a.rnxp);
  float taper = 1.0f;
  if (k > a.nz) {
    const float d = dist_to_boundary(k, a.nz, a.nzp);
    taper = fmaxf(__fsub_rn(1.0f, __fmul_rn(d, d)), 0.0f);
  }
  const bool tap = k > a.nz;
  for (int x = lane; x < cnxp; x += 32) {
    float2 v = r[x];
    const int i = 2 * x;
    if (i < a.nxp) {
      v.x = __fdiv_rn(v.x, a.sq);
      if (tap) v.x = __fmul_rn(v.x, taper);
    }
    if (i + 1 < a.nxp) {
      v.y = __fdiv_rn(v.y, a.sq);
      if (tap) v.y = __fmul_rn(v.y, taper);
    }
    r[x] = v;
  }
}

// The row padding (x >= nxp) set aside before the passes, one thread per row.
__global__ void __launch_bounds__(kThreads) k_div_save_pads(const __grid_constant__ DivPassArgs a) {
  const long long row = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= (long long)a.nyp * a.nzp) return;
  const int npad = a.rnxp - a.nxp;
  const float *src = a.grid + row * a.rnxp + a.nxp;
  for (int q = 0; q < npad; ++q) a.pads[row * npad + q] = src[q];
}

// After the inverse pass: value / sqrt(nzp) (:712-715); padding restored.
__global__ void __launch_bounds__(kThreads) k_div_post(const __grid_constant__ DivPassArgs a) {
  const int row = blockIdx.x * kRowsPerBlock + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (row >= a.nyp * a.nzp) return;
  const int cnxp = a.rnxp / 2, npad = a.rnxp - a.nxp;
  float2 *r = reinterpret_cast<float2 *>(a.grid + (long long)row * a.rnxp);
  const float *pad = a.pads + (long long)row * npad;
  for (int x = lane; x < cnxp; x += 32) {
    float2 v = r[x];
    const int i = 2 * x;
    v.x = i < a.nxp ? __fdiv_rn(v.x, a.sq) : pad[i - a.nxp];
    v.y = i + 1 < a.nxp ? __fdiv_rn(v.y, a.sq) : pad[i + 1 - a.nxp];
    r[x] = v;
  }
}

// Per trace: the frequency step of its bins and its stretch
// (src/crava.cpp:663-667).
__global__ void __launch_bounds__(kThreads) k_div_traces(const double *__restrict__ rel_thick, int n, int nz,
                                                        int nzp, double lz, double *df, float *sf) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const double relT = rel_thick[t];
  df[t] = (double)nz * 1000.0 / (relT * lz * (double)nzp);
  sf[t] = (float)(relT * (double)1.0f);  // relThick x getLocalStretch (1 for 1-D wavelets)
}

// ----------------------------------------------------------------- filter
struct DivFilterArgs {
  float2 *grid;               // complex view after the forward z pass
  const float2 *W, *E3;       // this angle's tables
  const float *tau2;
  const DivScalars *sc;
  const double *df;           // [nyp][nxp] frequency step of each trace
  const float *sf;            // [nyp][nxp] stretch of each trace
  const float *shift, *gain;  // [ny][nx] of this angle, or null
  int nxp, nyp, nzp, cnxp, nx, ny, nz;
  double lz;
  float dz, low_cut, high_cut, wnc;
};

// Mirrored simbox index of a padded trace (src/crava.cpp:622-640).
__device__ __forceinline__ int mirror(int i, int n, int np) {
  if (i > 3 * n - 1) i = 0;
  if (i > (np + n) / 2) i = np - i;
  if (i >= n) i = 2 * n - i - 1;
  return i;
}

// Bin m of a table as the local wavelet holds it: Wavelet1D::shiftAndScale
// (src/wavelet1D.cpp:539-561), ampMultiplier x value in float.
struct Local {
  float ishift, gain;
  bool on;
  double q1;  // ishift / nzp: the phase step per bin, in turns (set with on)
};

// The phase step of a local wavelet: one division per trace and bin where
// each rotation below would otherwise divide by nzp.  For a power-of-two
// nzp (the fused lengths) q1 * m equals ishift * m / nzp exactly; for other
// lengths it differs by at most an ulp of the double phase.
__device__ __forceinline__ void local_on(Local &L, float ishift, float gain, int nzp) {
  L.ishift = ishift;
  L.gain = gain;
  L.on = true;
  L.q1 = (double)ishift / (double)nzp;
}

// e^{-2 pi i ishift m / nzp}, the ampMultiplier phase of shiftAndScale.
// The reference evaluates cos / sin of 2 pi ishift m / nzp in double; here
// the phase in turns is reduced to (-1/2, 1/2] in double (ishift m / nzp for
// the float shift and integer bin) and the angle is evaluated in float,
// which keeps the rotation within a few 1e-7 while the per-(trace, bin)
// work stays off the FP64 pipe.
__device__ __forceinline__ float2 phase_rot(const Local &L, int m) {
  const double q = L.q1 * (double)m;
  const float f = (float)(q - rint(q));
  float sn, cs;
  sincospif(2.0f * f, &sn, &cs);
  return make_float2(cs, -sn);
}

// Bin m of the wavelet table as the local wavelet holds it, its rotation r
// (phase_rot(L, m)) given: gain x r x value in float.
__device__ __forceinline__ float2 local_bin_r(const float2 *tab, int m, const Local &L, float2 r) {
  const float2 v = __ldg(tab + m);
  if (!L.on) return v;
  const float ar = __fmul_rn(L.gain, r.x), ai = __fmul_rn(L.gain, r.y);
  return make_float2(__fsub_rn(__fmul_rn(ar, v.x), __fmul_rn(ai, v.y)),
                     __fadd_rn(__fmul_rn(ai, v.x), __fmul_rn(ar, v.y)));
}

// The normalised third difference of the local wavelet: the global one
// times 1/normF3, rotated by r (its gain cancels in the normalisation); the
// floats past nzp carry multiplyRAmpByConstant's RMISSING
// (src/wavelet.cpp:466-474).
__device__ __forceinline__ float2 local_e3_r(const float2 *E3, int m, int nzp, const Local &L, float inv, float2 r) {
  const float2 u = __ldg(E3 + m);
  float2 v = make_float2(__fmul_rn(u.x, inv), __fmul_rn(u.y, inv));
  if (L.on)
    v = make_float2(__fsub_rn(__fmul_rn(r.x, v.x), __fmul_rn(r.y, v.y)),
                    __fadd_rn(__fmul_rn(r.y, v.x), __fmul_rn(r.x, v.y)));
  if (m == nzp / 2) {
    if ((nzp & 1) == 0) v = make_float2(kMissing, kMissing);
    else v.y = kMissing;
  }
  return v;
}

__device__ __forceinline__ float2 local_e3(const float2 *E3, int m, int nzp, const Local &L, float inv) {
  return local_e3_r(E3, m, nzp, L, inv, L.on ? phase_rot(L, m) : make_float2(1.0f, 0.0f));
}

// |local_e3(E3, m)|^2: the rotation keeps the modulus, so it is needed
// only at the bin that carries RMISSING in one part (odd nzp).
__device__ __forceinline__ float local_e3_mag2(const float2 *E3, int m, int nzp, const Local &L, float inv) {
  if (m == nzp / 2 && (nzp & 1)) {
    const float2 v = local_e3(E3, m, nzp, L, inv);
    return __fadd_rn(__fmul_rn(v.x, v.x), __fmul_rn(v.y, v.y));
  }
  if (m == nzp / 2) return __fmul_rn(2.0f, __fmul_rn(kMissing, kMissing));
  const float2 u = __ldg(E3 + m);
  const float x = __fmul_rn(u.x, inv), y = __fmul_rn(u.y, inv);
  return __fadd_rn(__fmul_rn(x, x), __fmul_rn(y, y));
}

// Wavelet::getCAmp(k, scale) for k < cnzp (src/wavelet.cpp:327-385) of the
// local wavelet (w) and, when e3 is given, of its normalised third
// difference, from one pair of interpolation bins and one pair of
// rotations.
__device__ __forceinline__ void camp_scaled2(const float2 *W, const float2 *E3, int k, float scale, int nzp,
                                             const Local &L, float inv, float2 *w, float2 *e3) {
  const int cnzp = nzp / 2 + 1;
  const float omega = __fdividef((float)k, scale);
  float2 vw = make_float2(0.0f, 0.0f), ve = make_float2(0.0f, 0.0f);
  if (omega < (float)cnzp) {
    const int omL = (int)floorf(omega);
    int omU = omL + 1;
    if (omU >= cnzp) omU -= 1;
    const float dO = __fsub_rn(omega, (float)omL), dL = __fsub_rn(1.0f, dO);
    const float2 rL = L.on ? phase_rot(L, omL) : make_float2(1.0f, 0.0f);
    const float2 rU = L.on ? phase_rot(L, omU) : make_float2(1.0f, 0.0f);
    const float2 a = local_bin_r(W, omL, L, rL), b = local_bin_r(W, omU, L, rU);
    vw.x = __fadd_rn(__fmul_rn(a.x, dL), __fmul_rn(b.x, dO));
    vw.y = __fadd_rn(__fmul_rn(a.y, dL), __fmul_rn(b.y, dO));
    if (e3) {
      const float2 c = local_e3_r(E3, omL, nzp, L, inv, rL), d = local_e3_r(E3, omU, nzp, L, inv, rU);
      ve.x = __fadd_rn(__fmul_rn(c.x, dL), __fmul_rn(d.x, dO));
      ve.y = __fadd_rn(__fmul_rn(c.y, dL), __fmul_rn(d.y, dO));
    }
  }
  *w = make_float2(__fdividef(vw.x, scale), __fdividef(vw.y, scale));
  if (e3) *e3 = make_float2(__fdividef(ve.x, scale), __fdividef(ve.y, scale));
}

__device__ __forceinline__ float sq2(float2 v) { return __fadd_rn(__fmul_rn(v.x, v.x), __fmul_rn(v.y, v.y)); }

// computeAdjustmentFactor's value at bin k (src/crava.cpp:779-810) times
// the data bin, or 0 outside the band (:700-710).  The reference's float
// operations in its order, with its divisions as multiplications by the
// approximate reciprocal (__fdividef, 2 ulp): the spectra come from a
// different transform anyway, and the IEEE divisions made the kernel
// instruction-bound.
__device__ float2 adjust(const DivFilterArgs &a, int k, int i, int j, float2 d) {
  const long long tr = i + (long long)a.nxp * j;
  const double deltaF = __ldg(a.df + tr);
  if (!(deltaF * k < (double)a.high_cut && deltaF * k > (double)a.low_cut)) return make_float2(0.0f, 0.0f);
  Local L{0.0f, 1.0f, false, 0.0};
  if (a.shift || a.gain) {
    const int ii = mirror(i, a.nx, a.nxp), jj = mirror(j, a.ny, a.nyp);
    constexpr float kWellMissing = -999.0f;  // WELLMISSING, src/definitions.h:39
    float ts = 0.0f, g = 1.0f;
    // getLocalTimeshift / getLocalGainFactor read the grids only inside
    // them (src/wavelet.cpp:1143-1172); with much padding the mirrored
    // index can leave them
    if (ii >= 0 && ii < a.nx && jj >= 0 && jj < a.ny) {
      const long long o = ii + (long long)a.nx * jj;
      if (a.shift && a.shift[o] != kWellMissing) ts = a.shift[o];
      if (a.gain && a.gain[o] != kWellMissing) g = a.gain[o];
    }
    local_on(L, __fdiv_rn(ts, a.dz), g, a.nzp);
  }
  const float sf = __ldg(a.sf + tr);
  const DivScalars s = *a.sc;
  const float tolFac = 0.05f;
  float2 wLoc, e3Loc;
  camp_scaled2(a.W, a.E3, k, sf, a.nzp, L, s.e3_inv, &wLoc, &e3Loc);
  const float wLoc2 = sq2(wLoc);
  const float2 wGlob = __ldg(a.W + k);
  const float wGlob2 = sq2(wGlob);
  float sizeLoc = __fdividef(wLoc2, s.wn2);
  sizeLoc = __fadd_rn(sizeLoc, sq2(e3Loc));
  // |shifted and scaled W_k|^2 = gain^2 |W_k|^2 (the rotation keeps the modulus)
  const float g2 = L.on ? __fmul_rn(L.gain, L.gain) : 1.0f;
  float sizeGlob = __fdividef(__fmul_rn(g2, wGlob2), s.wn2);
  sizeGlob = __fadd_rn(sizeGlob, local_e3_mag2(a.E3, k, a.nzp, L, s.e3_inv));
  const float half = __fmul_rn(__fsub_rn(1.0f, a.wnc), 0.5f);
  float sigma2Loc = __fmul_rn(s.error_var, __fadd_rn(a.wnc, __fmul_rn(half, sizeLoc)));
  const float sigma2Glob = __fmul_rn(s.error_var, __fadd_rn(a.wnc, __fmul_rn(half, sizeGlob)));
  const float tau2 = __ldg(a.tau2 + k);
  float wGlob2Adj = wGlob2, wLoc2Adj = wLoc2;
  const float tm = __fmul_rn(tolFac, s.modW);
  if (wGlob2 < tm) wGlob2Adj = __fmul_rn(0.5f, __fadd_rn(wGlob2, tm));
  if (wLoc2 < tm) wLoc2Adj = __fmul_rn(0.5f, __fadd_rn(wLoc2, tm));
  if (wLoc2Adj < __fmul_rn(tolFac, wGlob2Adj)) {
    wLoc2Adj = __fmul_rn(0.5f, __fadd_rn(wLoc2, __fmul_rn(tolFac, wGlob2Adj)));
    sigma2Loc = __fmul_rn(sigma2Loc, __fdividef(wLoc2Adj, wLoc2));
  }
  const float den = __fadd_rn(__fmul_rn(tau2, wLoc2Adj), sigma2Loc);
  const float glob = __fdividef(wGlob2Adj, __fadd_rn(__fmul_rn(tau2, wGlob2), sigma2Glob));
  const float fr = __fdividef(__fdividef(wLoc.x, den), glob);
  const float fi = __fdividef(__fdividef(wLoc.y, den), glob);
  return make_float2(__fsub_rn(__fmul_rn(d.x, fr), __fmul_rn(d.y, fi)),
                     __fadd_rn(__fmul_rn(d.y, fr), __fmul_rn(d.x, fi)));
}

// One thread per (trace pair p, line j, bin k <= nzp/2): the pair's
// spectra A (trace 2p) and B (trace 2p+1) from z = a + i b at k and
// nzp - k, each adjusted, recombined.  Padding "traces" pass unchanged.
__global__ void __launch_bounds__(kThreads) k_div_filter(const __grid_constant__ DivFilterArgs a) {
  const long long plane = (long long)a.cnxp * a.nyp;
  const long long n = plane * (a.nzp / 2 + 1);
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n) return;
  const int k = (int)(idx / plane);
  const long long r = idx - (long long)k * plane;
  const int p = (int)(r % a.cnxp), j = (int)(r / a.cnxp);
  const int km = k == 0 ? 0 : a.nzp - k;
  const bool self = km == k;  // bin 0, and nzp/2 for even nzp
  float2 *zk = a.grid + r + (long long)k * plane;
  float2 *zm = a.grid + r + (long long)km * plane;
  const float2 Zk = *zk, Zm = *zm;
  // A = (Z_k + conj Z_m) / 2,  B = (Z_k - conj Z_m) / (2 i)
  float2 A = make_float2(0.5f * (Zk.x + Zm.x), 0.5f * (Zk.y - Zm.y));
  float2 B = make_float2(0.5f * (Zk.y + Zm.y), -0.5f * (Zk.x - Zm.x));
  const int ia = 2 * p, ib = 2 * p + 1;
  if (ia < a.nxp) {
    A = adjust(a, k, ia, j, A);
    if (self) A.y = 0.0f;  // the real inverse transform reads the real part here
  }
  if (ib < a.nxp) {
    B = adjust(a, k, ib, j, B);
    if (self) B.y = 0.0f;
  }
  *zk = make_float2(A.x - B.y, A.y + B.x);    // A + i B
  if (!self) *zm = make_float2(A.x + B.y, B.x - A.y);  // conj A + i conj B
}

// ------------------------------------------------------------- fused
// The whole per-stack step in one pass over HBM for the transform lengths
// compiled here: a CTA loads TX trace-pair columns of one y line (the
// pre-scale and taper applied on the way into shared memory), transforms
// them along z in place (the compile-time Stockham engine of the 3-D
// transforms), filters each pair's two spectra at k and nzp - k,
// transforms back and stores the traces it may write (the post-scale
// applied on the way out; other traces are not written at all).
// MODE 0: divideDataByScaleWavelet (every padded trace i < nxp);
// MODE 1: multiplyDataByScaleWaveletAndWriteToFile (simbox traces only).
struct FusedArgs {
  DivFilterArgs f;        // the division's filter inputs (MODE 0)
  const float2 *Wm;       // the multiply's wavelet spectrum (MODE 1)
  const float *sfm;       // the multiply's per-trace stretch (MODE 1)
  float *grid;            // real padded layout
  const float2 *tw;       // forward twiddles of length nzp
  float sq_in, sq_out;    // the divisors before and after
  int nx, ny, nxp, nyp, nzp, cnxp, rnxp, nz;
};

// The data bin times the conjugate of getCAmp(k, sf) of the trace's local
// wavelet (src/crava.cpp:852-865); the local shift and gain are read at
// the trace itself.
__device__ __forceinline__ float2 mul_conj(const FusedArgs &a, int k, int i, int j, float2 d) {
  Local L{0.0f, 1.0f, false, 0.0};
  if (a.f.shift || a.f.gain) {
    constexpr float kWellMissing = -999.0f;  // WELLMISSING, src/definitions.h:39
    const long long o = i + (long long)a.nx * j;
    float ts = 0.0f, g = 1.0f;
    if (a.f.shift && a.f.shift[o] != kWellMissing) ts = a.f.shift[o];
    if (a.f.gain && a.f.gain[o] != kWellMissing) g = a.f.gain[o];
    local_on(L, __fdiv_rn(ts, a.f.dz), g, a.nzp);
  }
  const float sf = __ldg(a.sfm + i + (long long)a.nxp * j);
  float2 w;
  camp_scaled2(a.Wm, nullptr, k, sf, a.nzp, L, 1.0f, &w, nullptr);
  return make_float2(__fadd_rn(__fmul_rn(d.x, w.x), __fmul_rn(d.y, w.y)),
                     __fsub_rn(__fmul_rn(d.y, w.x), __fmul_rn(d.x, w.y)));
}

template <int MODE>
__device__ __forceinline__ bool fused_trace(const FusedArgs &a, int i, int j) {
  return MODE == 0 ? i < a.nxp : (i < a.nx && j < a.ny);
}

template <int N, int TX, int MODE>
__global__ void __launch_bounds__(kThreads) k_div_fused(const __grid_constant__ FusedArgs a) {
  extern __shared__ float2 sm[];
  float2 *twl = sm;
  float2 *buf = twl + N;
  const int x0 = blockIdx.x * TX, j = blockIdx.y, tid = threadIdx.x;
  const long long plane = (long long)a.cnxp * a.nyp;
  float2 *col = reinterpret_cast<float2 *>(a.grid) + x0 + (long long)a.cnxp * j;
  for (int i = tid; i < N; i += kThreads) twl[i] = a.tw[i];
  for (int idx = tid; idx < TX * N; idx += kThreads) {
    const int t = idx % TX, m = idx / TX, p = x0 + t;
    float2 v = make_float2(0.0f, 0.0f);
    if (p < a.cnxp) {
      v = col[t + m * plane];
      float taper = 1.0f;
      if (MODE == 0 && m > a.nz) {
        const float d = dist_to_boundary(m, a.nz, a.nzp);
        taper = fmaxf(__fsub_rn(1.0f, __fmul_rn(d, d)), 0.0f);
      }
      if (fused_trace<MODE>(a, 2 * p, j)) {
        v.x = __fdiv_rn(v.x, a.sq_in);
        if (MODE == 0 && m > a.nz) v.x = __fmul_rn(v.x, taper);
      }
      if (fused_trace<MODE>(a, 2 * p + 1, j)) {
        v.y = __fdiv_rn(v.y, a.sq_in);
        if (MODE == 0 && m > a.nz) v.y = __fmul_rn(v.y, taper);
      }
    }
    buf[m * TX + t] = v;
  }
  __syncthreads();
  stockham_ip<N, -1, TX, 1, TX, kThreads>(buf, twl);
  for (int idx = tid; idx < TX * (N / 2 + 1); idx += kThreads) {
    const int t = idx % TX, k = idx / TX, p = x0 + t;
    if (p >= a.cnxp) continue;
    const int km = k == 0 ? 0 : N - k;
    const bool self = km == k;
    const float2 Zk = buf[k * TX + t], Zm = buf[km * TX + t];
    float2 A = make_float2(0.5f * (Zk.x + Zm.x), 0.5f * (Zk.y - Zm.y));
    float2 B = make_float2(0.5f * (Zk.y + Zm.y), -0.5f * (Zk.x - Zm.x));
    if (fused_trace<MODE>(a, 2 * p, j)) {
      A = MODE == 0 ? adjust(a.f, k, 2 * p, j, A) : mul_conj(a, k, 2 * p, j, A);
      if (self) A.y = 0.0f;
    }
    if (fused_trace<MODE>(a, 2 * p + 1, j)) {
      B = MODE == 0 ? adjust(a.f, k, 2 * p + 1, j, B) : mul_conj(a, k, 2 * p + 1, j, B);
      if (self) B.y = 0.0f;
    }
    buf[k * TX + t] = make_float2(A.x - B.y, A.y + B.x);
    if (!self) buf[km * TX + t] = make_float2(A.x + B.y, B.x - A.y);
  }
  __syncthreads();
  stockham_ip<N, 1, TX, 1, TX, kThreads>(buf, twl);
  float *rowbase = a.grid + (long long)a.rnxp * j;
  for (int idx = tid; idx < TX * N; idx += kThreads) {
    const int t = idx % TX, m = idx / TX, p = x0 + t;
    if (p >= a.cnxp) continue;
    const float2 v = buf[m * TX + t];
    const bool w0 = fused_trace<MODE>(a, 2 * p, j), w1 = fused_trace<MODE>(a, 2 * p + 1, j);
    float *dst = rowbase + 2 * p + (long long)a.rnxp * a.nyp * m;
    if (w0 && w1) {
      *reinterpret_cast<float2 *>(dst) = make_float2(__fdiv_rn(v.x, a.sq_out), __fdiv_rn(v.y, a.sq_out));
    } else {
      if (w0) dst[0] = __fdiv_rn(v.x, a.sq_out);
      if (w1) dst[1] = __fdiv_rn(v.y, a.sq_out);
    }
  }
}

// Launches the fused kernel when the transform length is compiled here;
// returns false (nothing launched) otherwise.
template <int MODE>
bool fused_launch(const FusedArgs &a, cudaStream_t s, int *rc) {
  constexpr int TX = 8;
  const dim3 grd((unsigned)((a.cnxp + TX - 1) / TX), (unsigned)a.nyp);
#define CRAVA_DIV_FUSED(NN)                                                         \
  if (a.nzp == NN) {                                                                \
    const size_t smem = sizeof(float2) * (NN + (size_t)TX * NN);                    \
    if ((*rc = func_smem((const void *)k_div_fused<NN, TX, MODE>, smem))) return true; \
    k_div_fused<NN, TX, MODE><<<grd, kThreads, smem, s>>>(a);                        \
    const cudaError_t e_ = cudaGetLastError();                                       \
    if (e_ != cudaSuccess) {                                                         \
      ::crava::set_last_error(e_, "kernel launch", __FILE__, __LINE__);              \
      *rc = CRAVA_GPU_ERR_CUDA;                                                      \
    } else {                                                                         \
      *rc = CRAVA_GPU_OK;                                                            \
    }                                                                                \
    return true;                                                                     \
  }
  CRAVA_DIV_FUSED(128) CRAVA_DIV_FUSED(256) CRAVA_DIV_FUSED(512)
#undef CRAVA_DIV_FUSED
  return false;
}

bool mis8(const void *q) { return !q || (reinterpret_cast<uintptr_t>(q) & 7u) != 0; }

}  // namespace

extern "C" int crava_gpu_divide_data_by_scale_wavelet(crava_gpu_ctx *c, float *const *data,
                                                      const float *cov_alpha, const double *rel_thick,
                                                      int nx, int ny, float dz, const float *shift,
                                                      const float *gain) {
  if (!c || !data || !cov_alpha || !rel_thick || !(dz > 0.0f)) return CRAVA_GPU_ERR_ARG;
  const Geom &g = c->g;
  const int nt = c->p.ntheta, nzp = g.nzp, cnzp = nzp / 2 + 1;
  if (nx < 1 || ny < 1 || nx > g.nxp || ny > g.nyp) return CRAVA_GPU_ERR_ARG;
  if (c->p.nz < 1 || c->p.nz > nzp) return CRAVA_GPU_ERR_ARG;
  for (int l = 0; l < nt; ++l) if (mis8(data[l])) return CRAVA_GPU_ERR_ARG;
  // shared memory of the spectra kernel: 2 nzp doubles, 5 nzp floats
  const size_t tab_smem = sizeof(double) * 2 * (size_t)nzp + sizeof(float) * 5 * (size_t)nzp;
  if (tab_smem > 227 * 1024) return CRAVA_GPU_ERR_ARG;
  DeviceGuard guard(c->device);
  const cudaStream_t s = c->stream;
  // device scratch (context-owned, grown on demand): tables, scalars, the
  // covAlpha column, relative thickness, shift and gain grids, row
  // padding, the context's wavelets and model constants
  const size_t nxy = (size_t)nx * ny, npad = (size_t)(g.rnxp - g.nxp) * g.nyp * g.nzp;
  char *buf = nullptr;
  size_t off = 0;
  auto take = [&](size_t n) { char *q = buf + off; off += (n + 15) & ~size_t(15); return q; };
  DivTables t;
  float *dshift, *dgain, *pads;
  double *rt, *tdf;
  float *tsf;
  char *dconst;
  // the context's wavelets, norms, A, var0 and theta packed for one upload
  const size_t o_wav = 0, o_norm = o_wav + ((sizeof(float) * nt * nzp + 15) & ~size_t(15));
  const size_t o_A = o_norm + ((sizeof(float) * nt + 15) & ~size_t(15));
  const size_t o_var = o_A + ((sizeof(float) * 3 * nt + 15) & ~size_t(15));
  const size_t o_th = o_var + ((sizeof(double) * 9 + 15) & ~size_t(15));
  const size_t nconst = o_th + sizeof(double) * nt * nt;
  auto carve = [&]() {
    off = 0;
    t.W = reinterpret_cast<float2 *>(take(sizeof(float2) * nt * cnzp));
    t.E3 = reinterpret_cast<float2 *>(take(sizeof(float2) * nt * cnzp));
    t.tau2 = reinterpret_cast<float *>(take(sizeof(float) * nt * cnzp));
    t.sc = reinterpret_cast<DivScalars *>(take(sizeof(DivScalars) * nt));
    rt = reinterpret_cast<double *>(take(sizeof(double) * g.nxp * g.nyp));
    tdf = reinterpret_cast<double *>(take(sizeof(double) * g.nxp * g.nyp));
    tsf = reinterpret_cast<float *>(take(sizeof(float) * g.nxp * g.nyp));
    dshift = shift ? reinterpret_cast<float *>(take(sizeof(float) * nt * nxy)) : nullptr;
    dgain = gain ? reinterpret_cast<float *>(take(sizeof(float) * nt * nxy)) : nullptr;
    pads = reinterpret_cast<float *>(take(sizeof(float) * (npad ? npad : 1)));
    dconst = take(nconst);
  };
  carve();  // sizes only (buf is null)
  const size_t bytes = off;
  if (c->div_bytes < bytes) {
    // the previous calls' work on the stream may still read the old buffer
    CRAVA_CUDA_TRY(cudaStreamSynchronize(s));
    cudaFree(c->div_buf);
    c->div_buf = nullptr;
    c->div_bytes = 0;
    if (cudaMalloc(reinterpret_cast<void **>(&c->div_buf), bytes) != cudaSuccess) return CRAVA_GPU_ERR_ALLOC;
    c->div_bytes = bytes;
  }
  buf = c->div_buf;
  carve();
  auto run = [&]() -> int {
    std::vector<char> hc(nconst);
    std::memcpy(hc.data() + o_wav, c->wavelet.data(), sizeof(float) * nt * nzp);
    if (!c->wnorm.empty()) std::memcpy(hc.data() + o_norm, c->wnorm.data(), sizeof(float) * nt);
    std::memcpy(hc.data() + o_A, c->A.data(), sizeof(float) * 3 * nt);
    std::memcpy(hc.data() + o_var, c->var0.data(), sizeof(double) * 9);
    std::memcpy(hc.data() + o_th, c->theta.data(), sizeof(double) * nt * nt);
    CRAVA_CUDA_TRY(cudaMemcpyAsync(dconst, hc.data(), nconst, cudaMemcpyHostToDevice, s));
    CRAVA_CUDA_TRY(cudaMemcpyAsync(rt, rel_thick, sizeof(double) * g.nxp * g.nyp, cudaMemcpyHostToDevice, s));
    if (shift) CRAVA_CUDA_TRY(cudaMemcpyAsync(dshift, shift, sizeof(float) * nt * nxy, cudaMemcpyHostToDevice, s));
    if (gain) CRAVA_CUDA_TRY(cudaMemcpyAsync(dgain, gain, sizeof(float) * nt * nxy, cudaMemcpyHostToDevice, s));
    DivConsts q{};
    q.wav = reinterpret_cast<const float *>(dconst + o_wav);
    q.wnorm = c->wnorm.empty() ? nullptr : reinterpret_cast<const float *>(dconst + o_norm);
    q.A = reinterpret_cast<const float *>(dconst + o_A);
    q.var0 = reinterpret_cast<const double *>(dconst + o_var);
    q.theta = reinterpret_cast<const double *>(dconst + o_th);
    q.cov_alpha = cov_alpha;
    q.col_stride = (long long)g.rnxp * g.nyp;
    q.nzp = nzp; q.nt = nt; q.nz = c->p.nz; q.lz = c->p.lz; q.dz = dz;
    q.low_cut = c->p.low_cut; q.high_cut = c->p.high_cut;
    int r2;
    if ((r2 = func_smem((const void *)k_div_spectra, tab_smem))) return r2;
    k_div_spectra<<<dim3(nt, (cnzp + kTabThreads - 1) / kTabThreads), kTabThreads, tab_smem, s>>>(q, t);
    CRAVA_LAUNCH_CHECK();
    k_div_scalars<<<nt, kTabThreads, 0, s>>>(q, t);
    CRAVA_LAUNCH_CHECK();
    DivPassArgs pa{};
    pa.pads = pads;
    pa.nxp = g.nxp; pa.nyp = g.nyp; pa.nzp = nzp; pa.rnxp = g.rnxp; pa.nz = c->p.nz;
    pa.sq = sqrtf((float)nzp);
    DivFilterArgs fa{};
    const int ntr = g.nxp * g.nyp;
    k_div_traces<<<(ntr + kThreads - 1) / kThreads, kThreads, 0, s>>>(rt, ntr, c->p.nz, nzp, c->p.lz, tdf, tsf);
    CRAVA_LAUNCH_CHECK();
    fa.df = tdf;
    fa.sf = tsf;
    fa.nxp = g.nxp; fa.nyp = g.nyp; fa.nzp = nzp; fa.cnxp = g.cnxp; fa.nx = nx; fa.ny = ny;
    fa.nz = c->p.nz; fa.lz = c->p.lz; fa.dz = dz;
    fa.low_cut = c->p.low_cut; fa.high_cut = c->p.high_cut; fa.wnc = c->p.wnc;
    const long long nfilt = (long long)g.cnxp * g.nyp * (nzp / 2 + 1);
    const long long rows = (long long)g.nyp * nzp;
    FusedArgs fu{};
    fu.tw = c->plans.z.tw;
    fu.sq_in = fu.sq_out = pa.sq;
    fu.nx = nx; fu.ny = ny; fu.nxp = g.nxp; fu.nyp = g.nyp; fu.nzp = nzp; fu.cnxp = g.cnxp;
    fu.rnxp = g.rnxp; fu.nz = c->p.nz;
    for (int l = 0; l < nt; ++l) {
      fa.W = t.W + (size_t)l * cnzp;
      fa.E3 = t.E3 + (size_t)l * cnzp;
      fa.tau2 = t.tau2 + (size_t)l * cnzp;
      fa.sc = t.sc + l;
      fa.shift = dshift ? dshift + (size_t)l * nxy : nullptr;
      fa.gain = dgain ? dgain + (size_t)l * nxy : nullptr;
      fu.f = fa;
      fu.grid = data[l];
      if (fused_launch<0>(fu, s, &r2)) {
        if (r2) return r2;
        continue;
      }
      pa.grid = data[l];
      k_div_save_pads<<<(unsigned)((rows + kThreads - 1) / kThreads), kThreads, 0, s>>>(pa);
      CRAVA_LAUNCH_CHECK();
      k_div_pre<<<(unsigned)((rows + kRowsPerBlock - 1) / kRowsPerBlock), kThreads, 0, s>>>(pa);
      CRAVA_LAUNCH_CHECK();
      if ((r2 = fft_cols_z(c->plans, reinterpret_cast<float2 *>(data[l]), -1, s))) return r2;
      fa.grid = reinterpret_cast<float2 *>(data[l]);
      k_div_filter<<<(unsigned)((nfilt + kThreads - 1) / kThreads), kThreads, 0, s>>>(fa);
      CRAVA_LAUNCH_CHECK();
      if ((r2 = fft_cols_z(c->plans, reinterpret_cast<float2 *>(data[l]), 1, s))) return r2;
      k_div_post<<<(unsigned)((rows + kRowsPerBlock - 1) / kRowsPerBlock), kThreads, 0, s>>>(pa);
      CRAVA_LAUNCH_CHECK();
    }
    return CRAVA_GPU_OK;
  };
  return run();
}

// ------------------------------------------------------ multiply back
// Crava::multiplyDataByScaleWaveletAndWriteToFile (src/crava.cpp:819-885)
// before its file write: the residual stacks back in the time domain, each
// simbox trace (i < nx, j < ny) times the conjugate spectrum of its
// stretched local wavelet.  The trace pairs are transformed in a scratch
// grid so that the traces the reference leaves alone stay bit for bit.
namespace {

struct MulPassArgs {
  const float *src;
  float *dst;
  int nx, ny, nxp, nyp, nzp, rnxp;
  float sq;  // the divisor of the pass
};

// grid -> scratch, every value / float(sqrt(float(nzp))) (:846-849)
__global__ void __launch_bounds__(kThreads) k_mul_pre(const __grid_constant__ MulPassArgs a) {
  const int row = blockIdx.x * kRowsPerBlock + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (row >= a.nyp * a.nzp) return;
  const int cnxp = a.rnxp / 2;
  const float2 *__restrict__ r = reinterpret_cast<const float2 *>(a.src + (long long)row * a.rnxp);
  float2 *__restrict__ w = reinterpret_cast<float2 *>(a.dst + (long long)row * a.rnxp);
  for (int x = lane; x < cnxp; x += 32) {
    const float2 v = r[x];
    w[x] = make_float2(__fdiv_rn(v.x, a.sq), __fdiv_rn(v.y, a.sq));
  }
}

// scratch -> grid for the simbox traces, / float(sqrt(double(nzp))) (:867-870)
__global__ void __launch_bounds__(kThreads) k_mul_post(const __grid_constant__ MulPassArgs a) {
  const int row = blockIdx.x * kRowsPerBlock + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (row >= a.nyp * a.nzp) return;
  const int j = row % a.nyp;
  if (j >= a.ny) return;
  const float *__restrict__ r = a.src + (long long)row * a.rnxp;
  float *__restrict__ w = a.dst + (long long)row * a.rnxp;
  for (int i = lane; i < a.nx; i += 32) w[i] = __fdiv_rn(r[i], a.sq);
}

struct MulFilterArgs {
  float2 *grid;               // scratch, complex view after the forward z pass
  const float2 *W;            // this angle's wavelet spectrum
  const float *sf;            // [nyp][nxp] float(relThick) x localStretch
  const float *shift, *gain;  // [ny][nx] of this angle, or null
  int nx, ny, nxp, nyp, nzp, cnxp;
  float dz;
};

// The data bin times the conjugate of getCAmp(k, sf) of the trace's local
// wavelet (src/crava.cpp:852-865).
__device__ __forceinline__ float2 mul_local(const MulFilterArgs &a, int k, int i, int j, float2 d) {
  Local L{0.0f, 1.0f, false, 0.0};
  if (a.shift || a.gain) {
    constexpr float kWellMissing = -999.0f;  // WELLMISSING, src/definitions.h:39
    const long long o = i + (long long)a.nx * j;
    float ts = 0.0f, g = 1.0f;
    if (a.shift && a.shift[o] != kWellMissing) ts = a.shift[o];
    if (a.gain && a.gain[o] != kWellMissing) g = a.gain[o];
    local_on(L, __fdiv_rn(ts, a.dz), g, a.nzp);
  }
  const float sf = __ldg(a.sf + i + (long long)a.nxp * j);
  float2 w;
  camp_scaled2(a.W, nullptr, k, sf, a.nzp, L, 1.0f, &w, nullptr);
  return make_float2(__fadd_rn(__fmul_rn(d.x, w.x), __fmul_rn(d.y, w.y)),
                     __fsub_rn(__fmul_rn(d.y, w.x), __fmul_rn(d.x, w.y)));
}

// One thread per (trace pair, line, bin k <= nzp/2), as k_div_filter;
// traces outside the simbox pass unchanged (they are not written back).
__global__ void __launch_bounds__(kThreads) k_mul_filter(const __grid_constant__ MulFilterArgs a) {
  const long long plane = (long long)a.cnxp * a.nyp;
  const long long n = plane * (a.nzp / 2 + 1);
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n) return;
  const int k = (int)(idx / plane);
  const long long r = idx - (long long)k * plane;
  const int p = (int)(r % a.cnxp), j = (int)(r / a.cnxp);
  if (j >= a.ny || 2 * p >= a.nx) return;
  const int km = k == 0 ? 0 : a.nzp - k;
  const bool self = km == k;
  float2 *zk = a.grid + r + (long long)k * plane;
  float2 *zm = a.grid + r + (long long)km * plane;
  const float2 Zk = *zk, Zm = *zm;
  float2 A = make_float2(0.5f * (Zk.x + Zm.x), 0.5f * (Zk.y - Zm.y));
  float2 B = make_float2(0.5f * (Zk.y + Zm.y), -0.5f * (Zk.x - Zm.x));
  A = mul_local(a, k, 2 * p, j, A);
  if (self) A.y = 0.0f;  // the real inverse transform reads the real part here
  if (2 * p + 1 < a.nx) {
    B = mul_local(a, k, 2 * p + 1, j, B);
    if (self) B.y = 0.0f;
  }
  *zk = make_float2(A.x - B.y, A.y + B.x);
  if (!self) *zm = make_float2(A.x + B.y, B.x - A.y);
}

__global__ void __launch_bounds__(kThreads) k_mul_traces(const double *__restrict__ rel_thick, int n, float *sf) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) sf[t] = __fmul_rn((float)rel_thick[t], 1.0f);  // getLocalStretch = 1 for 1-D wavelets
}

}  // namespace

namespace crava {

// Every simbox trace (x < nx, y < ny) of each grid[l] (real domain, or the
// spectrum when inverse_first, which is transformed back first) multiplied
// in the Fourier domain by the conjugate of its local wavelet's getCAmp(k,
// sf): the trace divided by pre_div, transformed, filtered, transformed
// back and divided by post_div.  Other traces are not touched.
int multiply_local_wavelet(crava_gpu_ctx *c, float *const *resid, const double *rel_thick, int nx, int ny,
                           float dz, const float *shift, const float *gain, float pre_div, float post_div,
                           bool inverse_first) {
  if (!c || !resid || !rel_thick || !(dz > 0.0f)) return CRAVA_GPU_ERR_ARG;
  const Geom &g = c->g;
  const int nt = c->p.ntheta, nzp = g.nzp, cnzp = nzp / 2 + 1;
  if (nx < 1 || ny < 1 || nx > g.nxp || ny > g.nyp) return CRAVA_GPU_ERR_ARG;
  for (int l = 0; l < nt; ++l) if (mis8(resid[l])) return CRAVA_GPU_ERR_ARG;
  const size_t tab_smem = sizeof(double) * 2 * (size_t)nzp + sizeof(float) * 5 * (size_t)nzp;
  if (tab_smem > 227 * 1024) return CRAVA_GPU_ERR_ARG;
  DeviceGuard guard(c->device);
  const cudaStream_t s = c->stream;
  const size_t nxy = (size_t)nx * ny;
  const bool fused_len = nzp == 128 || nzp == 256 || nzp == 512;  // k_div_fused lengths
  char *buf = nullptr;
  size_t off = 0;
  auto take = [&](size_t n) { char *q = buf + off; off += (n + 15) & ~size_t(15); return q; };
  DivTables t;
  float *dshift, *dgain, *tsf, *scratch;
  double *rt;
  char *dconst;
  const size_t o_wav = 0, o_norm = o_wav + ((sizeof(float) * nt * nzp + 15) & ~size_t(15));
  const size_t o_A = o_norm + ((sizeof(float) * nt + 15) & ~size_t(15));
  const size_t o_var = o_A + ((sizeof(float) * 3 * nt + 15) & ~size_t(15));
  const size_t o_th = o_var + ((sizeof(double) * 9 + 15) & ~size_t(15));
  const size_t nconst = o_th + sizeof(double) * nt * nt;
  auto carve = [&]() {
    off = 0;
    t.W = reinterpret_cast<float2 *>(take(sizeof(float2) * nt * cnzp));
    t.E3 = reinterpret_cast<float2 *>(take(sizeof(float2) * nt * cnzp));
    t.tau2 = reinterpret_cast<float *>(take(sizeof(float) * nt * cnzp));
    t.sc = reinterpret_cast<DivScalars *>(take(sizeof(DivScalars) * nt));
    rt = reinterpret_cast<double *>(take(sizeof(double) * g.nxp * g.nyp));
    tsf = reinterpret_cast<float *>(take(sizeof(float) * g.nxp * g.nyp));
    dshift = shift ? reinterpret_cast<float *>(take(sizeof(float) * nt * nxy)) : nullptr;
    dgain = gain ? reinterpret_cast<float *>(take(sizeof(float) * nt * nxy)) : nullptr;
    dconst = take(nconst);
    scratch = fused_len ? nullptr : reinterpret_cast<float *>(take(sizeof(float) * g.rsize));
  };
  carve();  // sizes only (buf is null)
  const size_t bytes = off;
  if (c->div_bytes < bytes) {
    CRAVA_CUDA_TRY(cudaStreamSynchronize(s));
    cudaFree(c->div_buf);
    c->div_buf = nullptr;
    c->div_bytes = 0;
    if (cudaMalloc(reinterpret_cast<void **>(&c->div_buf), bytes) != cudaSuccess) return CRAVA_GPU_ERR_ALLOC;
    c->div_bytes = bytes;
  }
  buf = c->div_buf;
  carve();
  std::vector<char> hc(nconst);
  std::memcpy(hc.data() + o_wav, c->wavelet.data(), sizeof(float) * nt * nzp);
  if (!c->wnorm.empty()) std::memcpy(hc.data() + o_norm, c->wnorm.data(), sizeof(float) * nt);
  std::memcpy(hc.data() + o_A, c->A.data(), sizeof(float) * 3 * nt);
  std::memcpy(hc.data() + o_var, c->var0.data(), sizeof(double) * 9);
  std::memcpy(hc.data() + o_th, c->theta.data(), sizeof(double) * nt * nt);
  CRAVA_CUDA_TRY(cudaMemcpyAsync(dconst, hc.data(), nconst, cudaMemcpyHostToDevice, s));
  CRAVA_CUDA_TRY(cudaMemcpyAsync(rt, rel_thick, sizeof(double) * g.nxp * g.nyp, cudaMemcpyHostToDevice, s));
  if (shift) CRAVA_CUDA_TRY(cudaMemcpyAsync(dshift, shift, sizeof(float) * nt * nxy, cudaMemcpyHostToDevice, s));
  if (gain) CRAVA_CUDA_TRY(cudaMemcpyAsync(dgain, gain, sizeof(float) * nt * nxy, cudaMemcpyHostToDevice, s));
  DivConsts q{};
  q.wav = reinterpret_cast<const float *>(dconst + o_wav);
  q.wnorm = nullptr;
  q.A = reinterpret_cast<const float *>(dconst + o_A);
  q.var0 = reinterpret_cast<const double *>(dconst + o_var);
  q.theta = reinterpret_cast<const double *>(dconst + o_th);
  q.cov_alpha = nullptr;  // the wavelet spectrum only
  q.col_stride = 0;
  q.nzp = nzp; q.nt = nt; q.nz = c->p.nz; q.lz = c->p.lz; q.dz = dz;
  q.low_cut = c->p.low_cut; q.high_cut = c->p.high_cut;
  int rc;
  if ((rc = func_smem((const void *)k_div_spectra, tab_smem))) return rc;
  k_div_spectra<<<dim3(nt, (cnzp + kTabThreads - 1) / kTabThreads), kTabThreads, tab_smem, s>>>(q, t);
  CRAVA_LAUNCH_CHECK();
  const int ntr = g.nxp * g.nyp;
  k_mul_traces<<<(ntr + kThreads - 1) / kThreads, kThreads, 0, s>>>(rt, ntr, tsf);
  CRAVA_LAUNCH_CHECK();
  const long long rows = (long long)g.nyp * nzp;
  const long long nfilt = (long long)g.cnxp * g.nyp * (nzp / 2 + 1);
  MulFilterArgs fa{};
  fa.sf = tsf;
  fa.nx = nx; fa.ny = ny; fa.nxp = g.nxp; fa.nyp = g.nyp; fa.nzp = nzp; fa.cnxp = g.cnxp; fa.dz = dz;
  fa.grid = reinterpret_cast<float2 *>(scratch);
  for (int l = 0; l < nt; ++l) {
    // seisData_[l]->invFFTInPlace() (:844)
    if (inverse_first && (rc = pass_inverse(c, resid[l], CRAVA_GRID_DATA))) return rc;
    if (fused_len) {
      FusedArgs fu{};
      fu.Wm = t.W + (size_t)l * cnzp;
      fu.sfm = tsf;
      fu.f.shift = dshift ? dshift + (size_t)l * nxy : nullptr;
      fu.f.gain = dgain ? dgain + (size_t)l * nxy : nullptr;
      fu.f.dz = dz;
      fu.grid = resid[l];
      fu.tw = c->plans.z.tw;
      fu.sq_in = pre_div;
      fu.sq_out = post_div;
      fu.nx = nx; fu.ny = ny; fu.nxp = g.nxp; fu.nyp = g.nyp; fu.nzp = nzp; fu.cnxp = g.cnxp;
      fu.rnxp = g.rnxp; fu.nz = c->p.nz;
      fused_launch<1>(fu, s, &rc);
      if (rc) return rc;
      continue;
    }
    MulPassArgs pa{resid[l], scratch, nx, ny, g.nxp, g.nyp, nzp, g.rnxp, pre_div};
    k_mul_pre<<<(unsigned)((rows + kRowsPerBlock - 1) / kRowsPerBlock), kThreads, 0, s>>>(pa);
    CRAVA_LAUNCH_CHECK();
    if ((rc = fft_cols_z(c->plans, reinterpret_cast<float2 *>(scratch), -1, s))) return rc;
    fa.W = t.W + (size_t)l * cnzp;
    fa.shift = dshift ? dshift + (size_t)l * nxy : nullptr;
    fa.gain = dgain ? dgain + (size_t)l * nxy : nullptr;
    k_mul_filter<<<(unsigned)((nfilt + kThreads - 1) / kThreads), kThreads, 0, s>>>(fa);
    CRAVA_LAUNCH_CHECK();
    if ((rc = fft_cols_z(c->plans, reinterpret_cast<float2 *>(scratch), 1, s))) return rc;
    MulPassArgs pb{scratch, resid[l], nx, ny, g.nxp, g.nyp, nzp, g.rnxp, post_div};
    k_mul_post<<<(unsigned)((rows + kRowsPerBlock - 1) / kRowsPerBlock), kThreads, 0, s>>>(pb);
    CRAVA_LAUNCH_CHECK();
  }
  return CRAVA_GPU_OK;
}

}  // namespace crava

extern "C" int crava_gpu_multiply_data_by_scale_wavelet(crava_gpu_ctx *c, float *const *resid,
                                                       const double *rel_thick, int nx, int ny, float dz,
                                                       const float *shift, const float *gain) {
  // rData[k] / sqrt(float nzp) before, / sqrt(double nzp) after (src/crava.cpp:853, 871)
  if (!c) return CRAVA_GPU_ERR_ARG;
  return crava::multiply_local_wavelet(c, resid, rel_thick, nx, ny, dz, shift, gain, sqrtf((float)c->g.nzp),
                                       (float)sqrt((double)c->g.nzp), true);
}
