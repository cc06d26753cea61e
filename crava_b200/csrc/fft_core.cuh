// fft_core.cuh -- small-radix butterflies and the shared-memory Stockham
// autosort engine used by every transform kernel.
//
// A line of length n = r_0 r_1 ... r_{s-1} is transformed by s radix-r
// stages; stage t reads the line with stride n/r and writes with stride Ns
// (the product of the radices already done), so the result comes out in
// natural order with no bit-reversal pass (Stockham autosort).  DIR = -1 is
// the forward transform (e^{-2 pi i k n / N}, FFTW_FORWARD), +1 the inverse;
// both are unnormalised.
#pragma once

#include "common.cuh"

namespace crava {

template <int DIR>
__device__ __forceinline__ float2 mul_dir_i(float2 a) {  // a * (DIR * i)
  return DIR < 0 ? make_float2(a.y, -a.x) : make_float2(-a.y, a.x);
}

template <int R, int DIR>
struct Dft;

template <int DIR>
struct Dft<2, DIR> {
  static __device__ __forceinline__ void run(float2 *v) {
    float2 a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  }
};

template <int DIR>
struct Dft<4, DIR> {
  static __device__ __forceinline__ void run(float2 *v) {
    float2 s02 = cadd(v[0], v[2]), d02 = csub(v[0], v[2]);
    float2 s13 = cadd(v[1], v[3]), d13 = mul_dir_i<DIR>(csub(v[1], v[3]));
    v[0] = cadd(s02, s13);
    v[2] = csub(s02, s13);
    v[1] = cadd(d02, d13);
    v[3] = csub(d02, d13);
  }
};

template <int DIR>
struct Dft<8, DIR> {
  static __device__ __forceinline__ void run(float2 *v) {
    float2 e[4] = {v[0], v[2], v[4], v[6]};
    float2 o[4] = {v[1], v[3], v[5], v[7]};
    Dft<4, DIR>::run(e);
    Dft<4, DIR>::run(o);
    const float h = 0.70710678118654752440f;
    // o[q] *= W8^q, W8 = e^{DIR i pi/4}
    float2 o1 = make_float2(h * (o[1].x - DIR * o[1].y), h * (o[1].y + DIR * o[1].x));
    float2 o2 = mul_dir_i<DIR>(o[2]);
    float2 o3 = make_float2(h * (-o[3].x - DIR * o[3].y), h * (-o[3].y + DIR * o[3].x));
    v[0] = cadd(e[0], o[0]);
    v[4] = csub(e[0], o[0]);
    v[1] = cadd(e[1], o1);
    v[5] = csub(e[1], o1);
    v[2] = cadd(e[2], o2);
    v[6] = csub(e[2], o2);
    v[3] = cadd(e[3], o3);
    v[7] = csub(e[3], o3);
  }
};

// Odd prime radix by the symmetric pairing a_k = v_k + v_{R-k},
// b_k = v_k - v_{R-k}: X_q = v_0 + sum_k cos(2 pi k q/R) a_k
//                          + DIR i sum_k sin(2 pi k q/R) b_k, X_{R-q} = conj-pair.
template <int R>
struct OddConst;
template <>
struct OddConst<3> {
  static __device__ __forceinline__ float c(int m) { return -0.5f; }
  static __device__ __forceinline__ float s(int m) { return 0.86602540378443864676f; }
};
template <>
struct OddConst<5> {
  static __device__ __forceinline__ float c(int m) {
    // cos(2 pi m / 5), m = 1..4
    return (m == 1 || m == 4) ? 0.30901699437494742410f : -0.80901699437494742410f;
  }
  static __device__ __forceinline__ float s(int m) {
    return m == 1 ? 0.95105651629515357212f
         : m == 2 ? 0.58778525229247312917f
         : m == 3 ? -0.58778525229247312917f
                  : -0.95105651629515357212f;
  }
};
template <>
struct OddConst<7> {
  static __device__ __forceinline__ float c(int m) {
    m %= 7;
    return (m == 1 || m == 6) ? 0.62348980185873353053f
         : (m == 2 || m == 5) ? -0.22252093395631440429f
                              : -0.90096886790241912624f;
  }
  static __device__ __forceinline__ float s(int m) {
    m %= 7;
    return m == 1 ? 0.78183148246802980871f
         : m == 2 ? 0.97492791218182360702f
         : m == 3 ? 0.43388373911755812048f
         : m == 4 ? -0.43388373911755812048f
         : m == 5 ? -0.97492791218182360702f
                  : -0.78183148246802980871f;
  }
};

template <int R, int DIR>
struct DftOdd {
  static __device__ __forceinline__ void run(float2 *v) {
    constexpr int H = (R - 1) / 2;
    float2 a[H], b[H];
    float2 sum = v[0];
#pragma unroll
    for (int k = 1; k <= H; ++k) {
      a[k - 1] = cadd(v[k], v[R - k]);
      b[k - 1] = csub(v[k], v[R - k]);
      sum = cadd(sum, a[k - 1]);
    }
    float2 out[R];
    out[0] = sum;
#pragma unroll
    for (int q = 1; q <= H; ++q) {
      float2 re = v[0], im = make_float2(0.f, 0.f);
#pragma unroll
      for (int k = 1; k <= H; ++k) {
        float c = OddConst<R>::c((k * q) % R), s = OddConst<R>::s((k * q) % R);
        re = make_float2(re.x + c * a[k - 1].x, re.y + c * a[k - 1].y);
        im = make_float2(im.x + s * b[k - 1].x, im.y + s * b[k - 1].y);
      }
      float2 t = mul_dir_i<DIR>(im);
      out[q] = cadd(re, t);
      out[R - q] = csub(re, t);
    }
#pragma unroll
    for (int q = 0; q < R; ++q) v[q] = out[q];
  }
};
template <int DIR> struct Dft<3, DIR> : DftOdd<3, DIR> {};
template <int DIR> struct Dft<5, DIR> : DftOdd<5, DIR> {};
template <int DIR> struct Dft<7, DIR> : DftOdd<7, DIR> {};

// One Stockham stage for every line held in shared memory.
//   src/dst : line l element m at  l*ls + m*es
//   tw      : e^{-2 pi i k/n}, k < n (shared memory)
//   mapping : lines_fastest -> task = j*nlines + l, else task = l*(n/R) + j
template <int R, int DIR>
__device__ __forceinline__ void stockham_stage(const float2 *__restrict__ src,
                                               float2 *__restrict__ dst, int n,
                                               int Ns, const float2 *tw,
                                               int nlines, int ls, int es,
                                               bool lines_fastest, int tid,
                                               int nthreads) {
  const int m = n / R;
  const int tasks = nlines * m;
  const int tstep = n / (Ns * R);
  for (int task = tid; task < tasks; task += nthreads) {
    int l, j;
    if (lines_fastest) { l = task % nlines; j = task / nlines; }
    else { j = task % m; l = task / m; }
    const float2 *s = src + l * ls;
    float2 v[R];
    const int base = j % Ns;
#pragma unroll
    for (int q = 0; q < R; ++q) v[q] = s[(j + q * m) * es];
    if (base != 0) {
      const int step = base * tstep;
#pragma unroll
      for (int q = 1; q < R; ++q) {
        float2 w = tw[(q * step) % n];
        if (DIR > 0) w.y = -w.y;
        v[q] = cmul(v[q], w);
      }
    }
    Dft<R, DIR>::run(v);
    const int idxD = (j / Ns) * Ns * R + base;
    float2 *d = dst + l * ls;
#pragma unroll
    for (int q = 0; q < R; ++q) d[(idxD + q * Ns) * es] = v[q];
  }
}

// Runs every stage; returns which buffer (0 = a, 1 = b) holds the result.
// The caller must __syncthreads() after filling `a` and `tw`.
template <int DIR>
__device__ int stockham_lines(float2 *a, float2 *b, const int *radix, int nr,
                              int n, const float2 *tw, int nlines, int ls,
                              int es, bool lines_fastest) {
  const int tid = threadIdx.x, nt = blockDim.x;
  float2 *src = a, *dst = b;
  int Ns = 1, which = 0;
  for (int st = 0; st < nr; ++st) {
    const int R = radix[st];
    switch (R) {
      case 8: stockham_stage<8, DIR>(src, dst, n, Ns, tw, nlines, ls, es, lines_fastest, tid, nt); break;
      case 4: stockham_stage<4, DIR>(src, dst, n, Ns, tw, nlines, ls, es, lines_fastest, tid, nt); break;
      case 2: stockham_stage<2, DIR>(src, dst, n, Ns, tw, nlines, ls, es, lines_fastest, tid, nt); break;
      case 3: stockham_stage<3, DIR>(src, dst, n, Ns, tw, nlines, ls, es, lines_fastest, tid, nt); break;
      case 5: stockham_stage<5, DIR>(src, dst, n, Ns, tw, nlines, ls, es, lines_fastest, tid, nt); break;
      default: stockham_stage<7, DIR>(src, dst, n, Ns, tw, nlines, ls, es, lines_fastest, tid, nt); break;
    }
    __syncthreads();
    Ns *= R;
    float2 *t = src; src = dst; dst = t;
    which ^= 1;
  }
  return which;
}

}  // namespace crava
