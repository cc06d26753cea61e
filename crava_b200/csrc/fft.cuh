// fft.cuh -- 3-D real<->complex transforms on the reference's padded layout.
#pragma once

#include "common.cuh"
#include "fft_core.cuh"
#include "fft_rr.cuh"

namespace crava {

// Plan for one line length: radix list and twiddle table e^{-2 pi i k/n}
// (n entries, float2) in device memory.
struct LinePlan {
  RadixList rl;
  float2 *tw = nullptr;
};

// Plans of one grid geometry.
struct FftPlans {
  Geom g;
  bool x_even = true;
  LinePlan x;        // length nxp/2 (even nxp) or nxp (odd)
  LinePlan y;        // length nyp
  LinePlan z;        // length nzp
  float2 *xpost = nullptr;  // e^{-2 pi i k/nxp}, k = 0..nxp/2 (even nxp)
  // column tile of the y and z passes: -1 default, 0 ping-pong pass,
  // 1 register-resident pass (lengths 64, 128, 256, 512), 8 or 16 columns
  // per CTA in the in-place pass (lengths with compiled kernels only; other
  // lengths use the generic pass), 2 (z only) the register-resident pass
  // with TMA tile loads where cols_z_tma_supported.  The default is the
  // TMA-fed pass where the fused x + y pass is in use and the grid allows
  // it, else the register-resident pass where it exists, else the in-place
  // pass.
  int tile_y = -1, tile_z = -1;
  // x pass of an even nxp: -1 default (register-resident where the half
  // length is 64..512), 0 the in-place pass, 1 register-resident
  int rows_x = -1;
  // x and y passes in one cluster kernel (plane.cu) where the geometry has
  // one: -1 default (on where the geometry has the kernel), 0 off, 1 on;
  // its twiddle tables (null where the geometry has none)
  int plane_xy = -1;
  float2 *twq = nullptr, *twy = nullptr;
};

// The fused x + y pass (plane.cu): geometries with a compiled kernel.
bool plane_xy_supported(const Geom &g);
int plane_xy_tables(const Geom &g, float2 **twq, float2 **twy);
// Forward (dir -1: src real -> dst spectrum in x and y, scaled) or inverse
// (dir +1: dst spectrum -> dst real, scaled, + addend) x and y passes.
int plane_xy(const FftPlans &p, const float *src, float *dst, int dir, float scale, const float *addend,
             cudaStream_t s);
// Whether the transforms of these plans use the fused x + y pass.
// Built in where the geometry has the kernel: alone it is slower than the
// separate register-resident x and y passes (129 / 113 us against 59 + 54 /
// 56 + 52 us per 256x256x512 grid, forward / inverse), but it moves two
// grids of HBM traffic instead of four, and in the unit, with the TMA-fed
// z pass and three transform lanes, it gave 5.23 ms against 5.40 ms.
inline bool use_plane_xy(const FftPlans &p) { return p.plane_xy != 0 && p.twq && p.twy; }

// Whether length n has compiled column kernels (tile choices 0, 8, 16).
bool cols_tunable(int n);
// Whether length n has register-resident kernels (column tile choice 1, and
// the x pass of nxp = 2 n).
bool cols_rr(int n);

bool radix_list(int n, RadixList *out);
int fft_plans_create(const Geom &g, FftPlans *p);
void fft_plans_destroy(FftPlans *p);

// In-place transforms of one grid with the FFTGrid scaling of `type`.
int fft3d_r2c(const FftPlans &p, float *grid, int type, cudaStream_t s);
// addend (optional): real grid added to the output (posterior mean of a realisation).
int fft3d_c2r(const FftPlans &p, float *grid, int type, cudaStream_t s,
              const float *addend = nullptr);

// Individual passes (used by the fused paths).
// src (forward only, optional): read the real input from src, write grid.
int fft_rows(const FftPlans &p, float *grid, int dir, float scale, cudaStream_t s,
             const float *addend = nullptr, const float *src = nullptr);
int fft_cols_y(const FftPlans &p, float2 *grid, int dir, cudaStream_t s);

// The band-gated covariance rule, applied by the forward z pass of a prior
// covariance grid as it stores the spectrum.  On a kz plane outside the
// inversion band (inv[kz] == 0) the per-bin loop of the reference only
// rewrites the prior covariance, |Re c / S0| S0 with Im 0
// (getNextParameterCovariance, src/seismicparametersholder.cpp:355-427;
// src/crava.cpp:1098-1147): done here, the solve visits the inverted planes
// alone and never reads or writes the band-gated bins.  mode 1: the FP64
// form's rule (the double expression rounded to float; for a finite c it
// equals sign(S0) |Re c| exactly, as the double error is far below half a
// float ulp, which needs c / S0 and its product with S0 to stay normal
// doubles: for any float c that holds for 1e-200 <= |S0| <= 1e200, and the
// host chooses mode 3, the double expression for every value, outside
// that range); mode 2: the mixed form's float operations.  A bin whose
// output is not finite sets its bit in nf_bits (and nf_any), so that the
// bins are counted once however many of the six grids hold a non-finite
// value (crava_gpu_stats.nonfinite_bins counts bins).
struct ZPrior {
  const int *inv = nullptr;     // [nzp] band flags; null: no epilogue
  double v = 0.0;               // this grid's Sigma0 entry
  // 1 FP64 form, |v| in [1e-200, 1e200] (or 0): sign(v) |c| for a finite c;
  // 3 FP64 form, other v: the double expression always; 2 mixed form
  int mode = 0;
  unsigned *nf_bits = nullptr;  // one bit per bin of the grid
  unsigned *nf_any = nullptr;
};

// The rare paths out of line: the FP64 form's double expression for a
// non-finite value, and the flagging of a non-finite output.
static __device__ __noinline__ float zprior_fp64_nonfinite(double v, float x) {
  const double d = (double)x;
  return (float)(v != 0.0 ? fabs(d / v) * v : fabs(d));
}
static __device__ __noinline__ void zprior_flag(unsigned *bits, unsigned *any, long long bin) {
  atomicOr(bits + (bin >> 5), 1u << (unsigned)(bin & 31));
  *(volatile unsigned *)any = 1u;
}

__device__ __forceinline__ float2 zprior_apply(const ZPrior &z, float2 x, long long bin) {
  float r;
  if (z.mode == 3) {
    r = zprior_fp64_nonfinite(z.v, x.x);
  } else if (z.mode == 1) {
    if (isfinite(x.x)) {
      const float a = fabsf(x.x);
      r = z.v != 0.0 ? (z.v < 0.0 ? -a : a) : a;
    } else {
      r = zprior_fp64_nonfinite(z.v, x.x);
    }
  } else {
    const float vf = (float)z.v;
    float y = x.x;
    if (z.v != 0.0) y = y / vf;
    r = fabsf(y) * vf;
  }
  if (!isfinite(r)) zprior_flag(z.nf_bits, z.nf_any, bin);
  return make_float2(r, 0.f);
}

// Bit b R + q set where the last stage's output register (b, q) of thread
// t lies on a band-gated kz plane: the band flags are read once per thread,
// not per tile.
template <int N, int E, int T>
__device__ __forceinline__ unsigned zprior_mask(const ZPrior &z, int t) {
  constexpr int S = CtRadix::count(N) - 1, R = CtRadix::at(N, S);
  static_assert(E <= 32, "one bit per register of a line");
  unsigned m = 0u;
  if (z.inv) {
#pragma unroll
    for (int b = 0; b < E / R; ++b)
#pragma unroll
      for (int q = 0; q < R; ++q)
        if (__ldg(z.inv + rr::stage_in<N, S, E, T>(t, b, q)) == 0) m |= 1u << (b * R + q);
  }
  return m;
}

// z pass; zp (forward only, optional): the band-gated covariance rule in
// its store (where z_prior_supported says the pass has it).
int fft_cols_z(const FftPlans &p, float2 *grid, int dir, cudaStream_t s, const ZPrior *zp = nullptr);
// Whether fft_cols_z applies a ZPrior under these plans for every grid of
// the geometry: the register-resident z pass and its TMA-fed form (lengths
// 64..512) do, the in-place and generic passes do not.
bool z_prior_supported(const FftPlans &p);

// z pass with TMA tile loads (cols_tma.cu; column tile choice 2): lengths
// 64..512, an even number of lines per z plane, a 16-byte aligned grid.
bool cols_z_tma_supported(const Geom &g, const void *data);
int cols_z_tma(const FftPlans &p, float2 *grid, int dir, cudaStream_t s, const ZPrior *zp = nullptr);
// Tile waits of the TMA z pass that hit their limit (device-wide, since the
// library was loaded; synchronous).
int tile_wait_timeouts(unsigned long long *out);

float forward_scale(const Geom &g, int type);
float inverse_scale(const Geom &g, int type);

}  // namespace crava
