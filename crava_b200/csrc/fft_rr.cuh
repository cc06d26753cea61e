// fft_rr.cuh -- register-resident transform passes (power-of-two lengths).
//
// The in-place passes of fft.cu stage every line in shared memory and run
// every radix stage shared memory -> registers -> shared memory, with the
// global load and store going through shared memory as well: about eight
// shared-memory operations per point and pass, and the passes are
// issue-bound at 50-69 % of the HBM copy rate.  Here each thread keeps its
// E points of a line in registers for the whole pass:
//
//   global -> registers, stage 0, registers -> shared, [sync],
//   shared -> registers, stage 1, ...,  last stage, registers -> global
//
// so a pass of S radix stages costs S - 1 shared-memory exchanges, and the
// first and last stages talk to HBM directly.  The arithmetic per butterfly
// is the Stockham stage of fft_core.cuh (same radices, same twiddle table,
// same butterflies), so the results equal the in-place passes bit for bit.
//
// Stage s of a line of N = R_0 ... R_{S-1} points (Ns = R_0 ... R_{s-1},
// M = N / R_s): butterfly j reads x[j + q M], q < R_s, multiplies by
// W_{Ns R}^{(j mod Ns) q}, and writes y[(j / Ns) Ns R + (j mod Ns) + q Ns].
// With E = max R_s points per thread and T = N / E threads per line,
// thread t takes the butterflies j = t + T b, b < E / R_s: its inputs are
// x[t + T (b + q E / R_s)], and in the last stage (Ns R = N) its outputs
// are y[t + T (b + q E / R)] -- the same stride-T set it loaded.
#pragma once

#include "fft_core.cuh"

namespace crava {
namespace rr {

__host__ __device__ constexpr int max_radix(int n) {
  int m = 0;
  for (int s = 0; s < CtRadix::count(n); ++s) m = CtRadix::at(n, s) > m ? CtRadix::at(n, s) : m;
  return m;
}
__host__ __device__ constexpr bool is_pow2(int n) { return n > 1 && (n & (n - 1)) == 0; }

// Lengths with register-resident kernels.
__host__ __device__ constexpr bool supported(int n) { return n == 64 || n == 128 || n == 256 || n == 512; }

// One radix stage on the thread's registers v[b R + q] (b < E / R).
template <int N, int S, int DIR, int E, int T>
__device__ __forceinline__ void stage_compute(float2 *v, const float2 *__restrict__ tw, int t) {
  constexpr int R = CtRadix::at(N, S);
  constexpr int NS = CtRadix::ns(N, S);
  constexpr int TSTEP = N / (NS * R);
#pragma unroll
  for (int b = 0; b < E / R; ++b) {
    float2 *w = v + b * R;
    if (NS > 1) {
      const int j = t + T * b;
      const int base = j % NS;
      if (base != 0) {
        const int step = base * TSTEP;
#pragma unroll
        for (int q = 1; q < R; ++q) {
          float2 x = tw[q * step];
          if (DIR > 0) x.y = -x.y;
          w[q] = cmul(w[q], x);
        }
      }
    }
    Dft<R, DIR>::run(w);
  }
}

// Per-stage twiddle tables.  Stage S >= 1 multiplies input q of butterfly
// j by W_N^{q (j mod NS) TSTEP}; reading those from the length-N table puts
// the threads of a warp on addresses that are multiples of TSTEP apart,
// most of them in the same bank.  The stage's own table holds the same
// values at q NS + (j mod NS), so the lanes of a warp, which differ in j,
// read consecutive entries: no bank conflicts, and the same floats (the
// outputs do not change).  Stage 0 (NS = 1) has no twiddles.  Used where it
// measured faster on B200: the TMA-fed z pass and the inverse x pass (the
// forward x pass and the y pass keep the length-N table).
template <int N>
struct TwStages {
  __host__ __device__ static constexpr int off(int s) {
    int o = 0;
    for (int i = 1; i < s; ++i) o += CtRadix::at(N, i) * CtRadix::ns(N, i);
    return o;
  }
  __host__ __device__ static constexpr int size() { return off(CtRadix::count(N)); }
};

// Shared-memory float2 slots of the per-stage tables (at least N, so the
// layouts that held the length-N table keep their offsets' alignment).
template <int N>
__host__ __device__ constexpr int tw_slots() {
  return TwStages<N>::size() > N ? TwStages<N>::size() : N;
}

// Fills the per-stage tables from the length-N table tw (one pass of the
// CTA's nth threads; the stage loop is unrolled at compile time, so an
// entry costs a shift, a mask and a multiply).
template <int N, int S = 1>
__device__ __forceinline__ void tw_stages_fill(float2 *tws, const float2 *__restrict__ tw, int tid, int nth) {
  if constexpr (S < CtRadix::count(N)) {
    constexpr int R = CtRadix::at(N, S), NS = CtRadix::ns(N, S), OFF = TwStages<N>::off(S);
    constexpr int TSTEP = N / (NS * R);
    for (int i = tid; i < R * NS; i += nth) tws[OFF + i] = tw[(i / NS) * (i % NS) * TSTEP];
    tw_stages_fill<N, S + 1>(tws, tw, tid, nth);
  }
}

// stage_compute with the twiddles from the per-stage tables.
template <int N, int S, int DIR, int E, int T>
__device__ __forceinline__ void stage_compute_st(float2 *v, const float2 *__restrict__ tws, int t) {
  constexpr int R = CtRadix::at(N, S);
  constexpr int NS = CtRadix::ns(N, S);
  constexpr int OFF = TwStages<N>::off(S);
#pragma unroll
  for (int b = 0; b < E / R; ++b) {
    float2 *w = v + b * R;
    if (NS > 1) {
      const int j = t + T * b;
      const int base = j % NS;
      if (base != 0) {
#pragma unroll
        for (int q = 1; q < R; ++q) {
          float2 x = tws[OFF + q * NS + base];
          if (DIR > 0) x.y = -x.y;
          w[q] = cmul(w[q], x);
        }
      }
    }
    Dft<R, DIR>::run(w);
  }
}

// Output element of register (b, q) after stage S.
template <int N, int S, int T>
__device__ __forceinline__ int stage_out(int t, int b, int q) {
  constexpr int R = CtRadix::at(N, S);
  constexpr int NS = CtRadix::ns(N, S);
  const int j = t + T * b;
  return (j / NS) * NS * R + (j % NS) + q * NS;
}

// Input element of register (b, q) for stage S.
template <int N, int S, int E, int T>
__device__ __forceinline__ constexpr int stage_in(int t, int b, int q) {
  constexpr int R = CtRadix::at(N, S);
  return t + T * (b + q * (E / R));
}

}  // namespace rr
}  // namespace crava
