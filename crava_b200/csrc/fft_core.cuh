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

// Radix 16 as 4 x 4: n = 4 n1 + n2, k = k1 + 4 k2:
//   Y[n2][k1] = DFT4_n1(x[4 n1 + n2]),  Y *= W16^(n2 k1),  X[k1 + 4 k2] = DFT4_n2(Y[.][k1]).
template <int DIR>
struct Dft<16, DIR> {
  static __device__ __forceinline__ float2 tw16(float2 a, int m) {
    // a * e^{DIR 2 pi i m / 16}, m in 1..9
    const float c1 = 0.92387953251128675613f, s1 = 0.38268343236508977173f;
    const float h = 0.70710678118654752440f;
    float c, sn;
    switch (m) {
      case 1: c = c1; sn = s1; break;
      case 2: c = h; sn = h; break;
      case 3: c = s1; sn = c1; break;
      case 4: c = 0.f; sn = 1.f; break;
      case 6: c = -h; sn = h; break;
      default: c = -c1; sn = -s1; break;  // m = 9
    }
    sn = DIR * sn;
    return make_float2(a.x * c - a.y * sn, a.x * sn + a.y * c);
  }
  static __device__ __forceinline__ void run(float2 *v) {
    float2 y[4][4];
#pragma unroll
    for (int n2 = 0; n2 < 4; ++n2) {
      float2 a[4] = {v[n2], v[4 + n2], v[8 + n2], v[12 + n2]};
      Dft<4, DIR>::run(a);
#pragma unroll
      for (int k1 = 0; k1 < 4; ++k1) y[n2][k1] = a[k1];
    }
#pragma unroll
    for (int n2 = 1; n2 < 4; ++n2)
#pragma unroll
      for (int k1 = 1; k1 < 4; ++k1) y[n2][k1] = tw16(y[n2][k1], n2 * k1);
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) {
      float2 b[4] = {y[0][k1], y[1][k1], y[2][k1], y[3][k1]};
      Dft<4, DIR>::run(b);
#pragma unroll
      for (int k2 = 0; k2 < 4; ++k2) v[k1 + 4 * k2] = b[k2];
    }
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

// Asynchronous global -> shared copies (cp.async, sm_80+): many copies per
// thread stay in flight until cp_async_wait_all().
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
// Waits until at most N of this thread's committed groups are pending.
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\n" ::);
  asm volatile("cp.async.wait_group 0;\n" ::);
}

// Division by a runtime constant d >= 1 as a multiply-high and a shift
// (round-up method of Granlund and Montgomery, "Division by invariant
// integers using multiplication", PLDI 1994), valid for n < 2^31.
struct FastDiv {
  uint32_t d, m, s;
};
__host__ __device__ inline FastDiv make_fastdiv(uint32_t d) {
  FastDiv f;
  f.d = d;
  f.s = 0;
  while ((1u << f.s) < d) ++f.s;
  f.m = (uint32_t)((((uint64_t)1 << 32) * (((uint64_t)1 << f.s) - d)) / d + 1);
  return f;
}
__device__ __forceinline__ uint32_t fdiv(uint32_t n, const FastDiv &f) {
  return (__umulhi(n, f.m) + n) >> f.s;
}

// One radix stage of a length-n line: R, the product Ns of the radices
// before it, m = n / R, the twiddle step n / (Ns R), and fast dividers.
struct Stage {
  int R, Ns, m, tstep;
  FastDiv fNs, fm;
};

// Radices of one line length, largest first (8, 4, 2, 3, 5, 7), with the
// per-stage constants precomputed on the host.
struct RadixList {
  int n;
  int nr;
  Stage st[16];
};

// One Stockham stage over `nlines` lines held in shared memory:
//   src line l element e at l*sls + e*ses, dst at l*dls + e*des.
// LF (lines fastest): consecutive threads take consecutive lines, which is
// conflict-free when the lines are adjacent words (element-major layouts);
// otherwise consecutive threads take consecutive butterflies of one line.
// Twiddles: tw[k] = e^{-2 pi i k / n}; the index q * base * tstep < n.
template <int R, int DIR, bool LF>
__device__ __forceinline__ void stockham_stage(const float2 *__restrict__ src, int sls, int ses,
                                               float2 *__restrict__ dst, int dls, int des,
                                               const Stage &sp, const float2 *__restrict__ tw,
                                               int nlines, const FastDiv &fl, int tid,
                                               int nthreads) {
  const int m = sp.m;
  const int tasks = nlines * m;
  for (int task = tid; task < tasks; task += nthreads) {
    int l, j;
    if (LF) { j = (int)fdiv((uint32_t)task, fl); l = task - j * nlines; }
    else { l = (int)fdiv((uint32_t)task, sp.fm); j = task - l * m; }
    const int jq = (int)fdiv((uint32_t)j, sp.fNs);
    const int base = j - jq * sp.Ns;
    const float2 *sl = src + l * sls;
    float2 v[R];
#pragma unroll
    for (int q = 0; q < R; ++q) v[q] = sl[(j + q * m) * ses];
    if (base != 0) {
      const int step = base * sp.tstep;
#pragma unroll
      for (int q = 1; q < R; ++q) {
        float2 w = tw[q * step];
        if (DIR > 0) w.y = -w.y;
        v[q] = cmul(v[q], w);
      }
    }
    Dft<R, DIR>::run(v);
    float2 *dl = dst + l * dls;
    const int idxD = jq * sp.Ns * R + base;
#pragma unroll
    for (int q = 0; q < R; ++q) dl[(idxD + q * sp.Ns) * des] = v[q];
  }
}

// All stages of a line transform, alternating between buffer a (layout
// als/aes) and b (bls/bes).  Returns 0 if the result is in a, 1 if in b.
// The caller synchronises before the call; every stage ends with a barrier.
template <int DIR, bool LF>
__device__ int stockham(float2 *a, int als, int aes, float2 *b, int bls, int bes,
                        const RadixList &rl, const float2 *tw, int nlines) {
  const int tid = threadIdx.x, nt = blockDim.x;
  const FastDiv fl = make_fastdiv((uint32_t)(nlines > 0 ? nlines : 1));
  float2 *src = a, *dst = b;
  int sls = als, ses = aes, dls = bls, des = bes;
  int which = 0;
  for (int s = 0; s < rl.nr; ++s) {
    const Stage &sp = rl.st[s];
    switch (sp.R) {
      case 8: stockham_stage<8, DIR, LF>(src, sls, ses, dst, dls, des, sp, tw, nlines, fl, tid, nt); break;
      case 4: stockham_stage<4, DIR, LF>(src, sls, ses, dst, dls, des, sp, tw, nlines, fl, tid, nt); break;
      case 2: stockham_stage<2, DIR, LF>(src, sls, ses, dst, dls, des, sp, tw, nlines, fl, tid, nt); break;
      case 3: stockham_stage<3, DIR, LF>(src, sls, ses, dst, dls, des, sp, tw, nlines, fl, tid, nt); break;
      case 5: stockham_stage<5, DIR, LF>(src, sls, ses, dst, dls, des, sp, tw, nlines, fl, tid, nt); break;
      default: stockham_stage<7, DIR, LF>(src, sls, ses, dst, dls, des, sp, tw, nlines, fl, tid, nt); break;
    }
    __syncthreads();
    float2 *t = src; src = dst; dst = t;
    int x = sls; sls = dls; dls = x;
    x = ses; ses = des; des = x;
    which ^= 1;
  }
  return which;
}

}  // namespace crava

namespace crava {

// ---------------------------------------------------------------------------
// Compile-time Stockham engine: the line length N, the number of lines NL
// and the strides are template constants, so every index, stride and
// twiddle step folds to constants (no runtime division).
// Radices: 8 while possible, then 4, then 2, then 3, 5, 7 (as radix_list).
// ---------------------------------------------------------------------------
struct CtRadix {
  // Radix sequence: 8 while possible, then 4, then 2, then 3, 5, 7; or, when
  // it takes fewer stages, 16 while possible first (e.g. 256 = 16 x 16).
  __host__ __device__ static constexpr int pick(int m, bool use16) {
    return (use16 && m % 16 == 0) ? 16
         : (m % 8 == 0) ? 8 : (m % 4 == 0) ? 4 : (m % 2 == 0) ? 2
         : (m % 3 == 0) ? 3 : (m % 5 == 0) ? 5 : (m % 7 == 0) ? 7 : m;
  }
  __host__ __device__ static constexpr int stages(int n, bool use16) {
    int m = n, c = 0;
    while (m > 1) { m /= pick(m, use16); ++c; }
    return c;
  }
  __host__ __device__ static constexpr bool use16(int n) { return stages(n, true) < stages(n, false); }
  __host__ __device__ static constexpr int at(int n, int s) {
    int m = n, r = 1;
    for (int i = 0; i <= s; ++i) { r = pick(m, use16(n)); m /= r; }
    return r;
  }
  __host__ __device__ static constexpr int count(int n) { return stages(n, use16(n)); }
  __host__ __device__ static constexpr int ns(int n, int s) {
    int p = 1;
    for (int i = 0; i < s; ++i) p *= at(n, i);
    return p;
  }
  __host__ __device__ static constexpr bool supported(int n) {
    int m = n;
    while (m % 2 == 0) m /= 2;
    while (m % 3 == 0) m /= 3;
    while (m % 5 == 0) m /= 5;
    while (m % 7 == 0) m /= 7;
    return m == 1 && n > 1;
  }
};
static_assert(CtRadix::count(256) == 2 && CtRadix::at(256, 0) == 16, "radix plan");
static_assert(CtRadix::count(128) == 2 && CtRadix::at(128, 1) == 8, "radix plan");
static_assert(CtRadix::count(512) == 3 && CtRadix::at(512, 0) == 8, "radix plan");

template <int N, int R, int NS, int DIR, bool LF, int NL, int SLS, int SES, int DLS, int DES>
__device__ __forceinline__ void ct_stage(const float2 *__restrict__ src, float2 *__restrict__ dst,
                                         const float2 *__restrict__ tw, int tid, int nth) {
  constexpr int M = N / R;
  constexpr int TASKS = NL * M;
  constexpr int TSTEP = N / (NS * R);
  for (int task = tid; task < TASKS; task += nth) {
    int l, j;
    if (LF) { l = task % NL; j = task / NL; }
    else { j = task % M; l = task / M; }
    const int base = j % NS;
    const float2 *sl = src + l * SLS + j * SES;
    float2 v[R];
#pragma unroll
    for (int q = 0; q < R; ++q) v[q] = sl[q * M * SES];
    if (NS > 1 && base != 0) {
      const int step = base * TSTEP;
#pragma unroll
      for (int q = 1; q < R; ++q) {
        float2 w = tw[q * step];
        if (DIR > 0) w.y = -w.y;
        v[q] = cmul(v[q], w);
      }
    }
    Dft<R, DIR>::run(v);
    float2 *dl = dst + l * DLS + ((j / NS) * NS * R + base) * DES;
#pragma unroll
    for (int q = 0; q < R; ++q) dl[q * NS * DES] = v[q];
  }
}

template <int N, int DIR, bool LF, int NL, int ALS, int AES, int BLS, int BES, int S>
struct CtStages {
  static __device__ __forceinline__ void run(float2 *a, float2 *b, const float2 *tw, int tid, int nth) {
    if constexpr (S < CtRadix::count(N)) {
      constexpr int R = CtRadix::at(N, S);
      constexpr int NS = CtRadix::ns(N, S);
      ct_stage<N, R, NS, DIR, LF, NL, ALS, AES, BLS, BES>(a, b, tw, tid, nth);
      __syncthreads();
      CtStages<N, DIR, LF, NL, BLS, BES, ALS, AES, S + 1>::run(b, a, tw, tid, nth);
    }
  }
};

// All stages; returns 0 if the result is in a, 1 if in b (odd stage count).
template <int N, int DIR, bool LF, int NL, int ALS, int AES, int BLS, int BES>
__device__ __forceinline__ int stockham_ct(float2 *a, float2 *b, const float2 *tw) {
  CtStages<N, DIR, LF, NL, ALS, AES, BLS, BES, 0>::run(a, b, tw, threadIdx.x, blockDim.x);
  return CtRadix::count(N) & 1;
}

}  // namespace crava

namespace crava {

// Element pitch (float2) of a TX-line in-place column buffer.  (A pitch of
// 9 for 8 lines removes the first stage's write conflicts but adds
// conflicts to every load and measured 20 % slower at 512 points.)
__host__ __device__ constexpr int cols_pitch(int tx) { return tx; }

// Row padding of a TX-line column buffer of length n: one spare row after
// every PADR rows (0: none).  With 8 lines (16 banks per row) the first
// stage of a power-of-two radix R writes rows R apart from the four
// butterflies a warp holds, all in the same 16 banks; a spare row every R
// rows would move every other butterfly to the other 16 banks.  Measured
// at 512 points it removes the conflicts but not the time (the pass is
// issue-bound and the row arithmetic costs what the conflicts did), so it
// is off.
__host__ __device__ constexpr int cols_padr(int, int) { return 0; }
// Physical row of logical row e (PADR a power of two or 0).
template <int PADR>
__host__ __device__ __forceinline__ constexpr int pad_row(int e) { return PADR ? e + e / PADR : e; }
// Rows a padded buffer of n elements needs.
__host__ __device__ constexpr int padded_rows(int n, int padr) { return padr ? n + n / padr : n; }

// In-place compile-time Stockham: each stage first reads every butterfly
// input of this thread into registers, synchronises, then writes the
// outputs into the same buffer.  Halves the shared memory of the
// ping-pong form.  NTH is the block size (compile-time); element e of a
// line sits at row pad_row<PADR>(e).
template <int N, int R, int NS, int DIR, int NL, int LS, int ES, int NTH, int PADR>
__device__ __forceinline__ void ct_stage_ip(float2 *buf, const float2 *__restrict__ tw, int tid) {
  constexpr int M = N / R;
  constexpr int TSTEP = N / (NS * R);
  static_assert(NTH % NL == 0, "block size must be a multiple of the line count");
  // Lines fastest: thread tid always works on line l = tid % NL; its
  // butterflies are j = j0 + i * JS.
  constexpr int JS = NTH / NL;
  constexpr int PER = (M + JS - 1) / JS;
  const int l = tid % NL;
  const int j0 = tid / NL;
  float2 *lb = buf + l * LS;
  float2 v[PER][R];
#pragma unroll
  for (int i = 0; i < PER; ++i) {
    const int j = j0 + i * JS;
    if (M % JS == 0 || j < M) {
#pragma unroll
      for (int q = 0; q < R; ++q) v[i][q] = lb[pad_row<PADR>(j + q * M) * ES];
    }
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < PER; ++i) {
    const int j = j0 + i * JS;
    if (M % JS == 0 || j < M) {
      const int base = j % NS;
      if (NS > 1 && base != 0) {
        const int step = base * TSTEP;
#pragma unroll
        for (int q = 1; q < R; ++q) {
          float2 w = tw[q * step];
          if (DIR > 0) w.y = -w.y;
          v[i][q] = cmul(v[i][q], w);
        }
      }
      Dft<R, DIR>::run(v[i]);
      const int e0 = (j - base) * R + base;
#pragma unroll
      for (int q = 0; q < R; ++q) lb[pad_row<PADR>(e0 + q * NS) * ES] = v[i][q];
    }
  }
  __syncthreads();
}

template <int N, int DIR, int NL, int LS, int ES, int NTH, int PADR, int S>
struct CtStagesIp {
  static __device__ __forceinline__ void run(float2 *buf, const float2 *tw, int tid) {
    if constexpr (S < CtRadix::count(N)) {
      ct_stage_ip<N, CtRadix::at(N, S), CtRadix::ns(N, S), DIR, NL, LS, ES, NTH, PADR>(buf, tw, tid);
      CtStagesIp<N, DIR, NL, LS, ES, NTH, PADR, S + 1>::run(buf, tw, tid);
    }
  }
};

// Transforms NL lines of length N in place (caller syncs before).
template <int N, int DIR, int NL, int LS, int ES, int NTH, int PADR = 0>
__device__ __forceinline__ void stockham_ip(float2 *buf, const float2 *tw) {
  CtStagesIp<N, DIR, NL, LS, ES, NTH, PADR, 0>::run(buf, tw, threadIdx.x);
}

}  // namespace crava
