// plane.cu -- the x and y passes of a 3-D transform in one kernel: one
// thread-block cluster per (grid, z-plane), the plane held in the CTAs'
// shared memory, so a transform moves 4 grids of HBM traffic (this pass
// and the z pass each read and write the grid once) instead of 6.
//
// A plane of NY rows of nxp = 2 NH reals is split over the CS CTAs of a
// cluster by rows: CTA r holds the NQ = NY / CS rows y = CS q + r.  The y
// transform of length NY = NQ CS factorises (ky = k1 + NQ k2):
//   Y[k1 + NQ k2] = sum_r W_CS^{r k2} [ W_NY^{r k1} sum_q x[CS q + r] W_NQ^{q k1} ],
// so each CTA first transforms its rows along x (the packed half-length
// R2C of the x pass), then along its own rows with NQ points and the
// twiddle W_NY^{r k1}; after a cluster barrier the last radix-CS stage
// runs across the CTAs: CTA r reads the CS values of its quarter of the
// k1 range from every CTA's shared memory (distributed shared memory) and
// writes the CS spectrum rows k1 + NQ k2 straight to HBM.  The inverse
// runs the same steps backwards: the radix-CS stage from HBM, its results
// pushed into the owning CTAs' shared memory, the NQ-point inverse along
// y, and the x C2R to HBM.
//
// The per-line arithmetic uses the register-resident Stockham stages of
// fft_rr.cuh.  The y factorisation differs from the separate y pass
// (radix CS first instead of the CtRadix list), so the results agree with
// the three-pass transforms to float rounding, not bit for bit.
//
// Replaces the x and y passes of FFTGrid::fftInPlace / invFFTInPlace
// (src/fftgrid.cpp:1803-1862); the scalings are fused as in fft.cu.
#include <cooperative_groups.h>
#include <math.h>

#include <vector>

#include "fft.cuh"
#include "fft_rr.cuh"

namespace cg = cooperative_groups;

namespace crava {

namespace {

// 288 threads: the y stage covers the cnxp = NH + 1 columns in two rounds
// (72 per round at 4 threads a column) instead of two full rounds and a
// third holding the Nyquist column alone; three CTAs per SM
constexpr int kPlaneThreads = 288;
constexpr int kPlaneMinBlocks = 3;
// items per thread whose HBM loads the inverse's radix-CS stage keeps in
// flight together
constexpr int kInvItems = 4;

struct PlaneArgs {
  const float *src;   // forward: real input planes (may equal dst)
  float *dst;         // forward: spectrum output; inverse: real output
  const float *add;   // inverse: real addend or null
  int rnxp, nyp, nplanes;
  float scale;
  const float2 *twx;   // NH-point table e^{-2 pi i k / NH}
  const float2 *post;  // e^{-2 pi i k / nxp}, k <= NH
  const float2 *twq;   // NQ-point table
  const float2 *twy;   // NY-point table e^{-2 pi i k / NY}
};

template <int NH, int NY, int CS>
struct PlaneCfg {
  static constexpr int NQ = NY / CS;
  static constexpr int CX = NH + 1;   // cnxp
  static constexpr int EX = rr::max_radix(NH), TX = NH / EX;   // x: points / threads per row
  static constexpr int R0X = CtRadix::at(NH, 0);
  static constexpr int EQ = rr::max_radix(NQ), TQ = NQ / EQ;  // y: points / threads per column
  // row pitch: the x exchange layout (one spare after every R0X) and the
  // CX outputs both fit; 8 mod 16 float2 keeps two rows per phase apart
  static constexpr int P0 = (NH + NH / R0X) > CX ? (NH + NH / R0X) : CX;
  static constexpr int P = P0 + ((8 - P0 % 16) + 16) % 16;
  static constexpr int QK = NQ / CS;  // k1 range of one CTA in the radix-CS stage
  static __host__ __device__ constexpr int physx(int e) { return e + e / R0X; }
  // tables, padded to an even float2 count so the plane buffer A starts on
  // a 16-byte boundary (16-byte cp.async copies land in it)
  static constexpr int TABN = NH + NH + 1 + NQ + NQ;
  static constexpr size_t tab = sizeof(float2) * (TABN + (TABN & 1));
  static constexpr size_t smem = tab + sizeof(float2) * (size_t)NQ * P;
};

// Barrier of a line's exchanges: a warp barrier where the line's threads
// lie in one warp (the x rows: TX consecutive threads, TX a power of two
// <= 32), the block barrier otherwise (the y columns: 4 threads a column,
// strided by the columns of a round).
template <bool WARP>
__device__ __forceinline__ void line_sync() {
  if constexpr (WARP) __syncwarp();
  else __syncthreads();
}

template <int N, int DIR, int E, int T, int S, bool WARP, typename IDX>
struct SmemStages {
  // stages S.. of an N-point line held as v (registers) with exchanges in
  // shared memory at idx(e); the caller syncs before the first call
  static __device__ __forceinline__ void run(float2 (&v)[E], float2 *buf, const float2 *tw, int t, bool act,
                                             IDX idx) {
    constexpr int R = CtRadix::at(N, S);
    if (act) rr::stage_compute<N, S, DIR, E, T>(v, tw, t);
    if constexpr (S + 1 < CtRadix::count(N)) {
      line_sync<WARP>();  // every thread has read this stage's inputs
      if (act) {
#pragma unroll
        for (int b = 0; b < E / R; ++b)
#pragma unroll
          for (int q = 0; q < R; ++q) buf[idx(rr::stage_out<N, S, T>(t, b, q))] = v[b * R + q];
      }
      line_sync<WARP>();
      constexpr int R2 = CtRadix::at(N, S + 1);
      if (act) {
#pragma unroll
        for (int b = 0; b < E / R2; ++b)
#pragma unroll
          for (int q = 0; q < R2; ++q) v[b * R2 + q] = buf[idx(rr::stage_in<N, S + 1, E, T>(t, b, q))];
      }
      SmemStages<N, DIR, E, T, S + 1, WARP, IDX>::run(v, buf, tw, t, act, idx);
    }
  }
};

// Register of position t + T m after the last stage of radix RL: the
// stage's inputs t + T (b + q E / RL) sit at register b RL + q.
template <int E, int RL>
__device__ __forceinline__ constexpr int last_reg(int m) {
  return (m % (E / RL)) * RL + m / (E / RL);
}

// ------------------------------------------------------------------ forward
template <int NH, int NY, int CS>
__global__ void __launch_bounds__(kPlaneThreads, kPlaneMinBlocks) k_plane_xy_fwd(const __grid_constant__ PlaneArgs a) {
  using C = PlaneCfg<NH, NY, CS>;
  constexpr int NQ = C::NQ, CX = C::CX, P = C::P, EX = C::EX, TX = C::TX, EQ = C::EQ, TQ = C::TQ;
  constexpr int R0X = C::R0X, SX = CtRadix::count(NH), RLX = CtRadix::at(NH, SX - 1);
  constexpr int R0Q = CtRadix::at(NQ, 0), SQ = CtRadix::count(NQ), RLQ = CtRadix::at(NQ, SQ - 1);
  cg::cluster_group cl = cg::this_cluster();
  extern __shared__ float4 sm4[];
  float2 *twx = reinterpret_cast<float2 *>(sm4);
  float2 *post = twx + NH;
  float2 *twq = post + NH + 1;
  float2 *twr = twq + NQ;  // W_NY^{r k1}, k1 < NQ
  float2 *A = twx + C::TABN + (C::TABN & 1);  // [NQ][P], 16-byte aligned
  const int tid = threadIdx.x, r = (int)cl.block_rank();
  for (int i = tid; i < NH; i += kPlaneThreads) twx[i] = a.twx[i];
  for (int i = tid; i <= NH; i += kPlaneThreads) post[i] = a.post[i];
  for (int i = tid; i < NQ; i += kPlaneThreads) {
    twq[i] = a.twq[i];
    twr[i] = a.twy[(r * i) % NY];
  }
  const int plane = blockIdx.x / CS;
  const long long pr = (long long)a.rnxp * a.nyp;  // floats per real plane
  const float *src = a.src + (long long)plane * pr;
  float2 *dst = reinterpret_cast<float2 *>(a.dst + (long long)plane * pr);

  // 1. x: the NQ rows of this CTA, TX threads per row, rounds of
  //    kPlaneThreads / TX rows.  Every round's input rows travel into A by
  //    cp.async before the first round computes (one commit group per
  //    round), so the HBM reads of a later round run under the arithmetic of
  //    the earlier one.  A row y starts on a 16-byte boundary when y is even
  //    (rnxp * 4 = 8 (NH + 1) bytes a row, NH + 1 odd); y = CS q + r has the
  //    parity of r, the same for every row of this CTA.  Even rows are
  //    copied as NH / 2 16-byte pairs into row[0 ..]; odd rows land one
  //    element further, row[1 ..]: element 0 by an 8-byte copy, then the
  //    pairs (1, 2) .. (NH - 1, NH) (element NH is the row's padding, inside
  //    the row) as 16-byte copies.  A grid that is not 16-byte aligned takes
  //    8-byte copies throughout.
  constexpr int RPR = kPlaneThreads / TX;  // rows per round
  constexpr int NRX = (NQ + RPR - 1) / RPR;
  static_assert(NRX <= 2, "the commit-group waits below cover two rounds");
  static_assert((P % 2) == 0 && NH + 1 < P, "16-byte aligned rows with room for the shifted landing");
  const bool wide = (reinterpret_cast<uintptr_t>(a.src) & 15u) == 0;
  const int off = (wide && (r & 1)) ? 1 : 0;  // landing offset of this CTA's rows
#pragma unroll
  for (int rd = 0; rd < NRX; ++rd) {
    const int q0 = rd * RPR, nr = NQ - q0 < RPR ? NQ - q0 : RPR;
    if (wide) {
      constexpr int TPR = NH / 2 + 1;  // tasks per row: the odd rows' single, then the pairs
      for (int i = tid; i < nr * TPR; i += kPlaneThreads) {
        const int q = q0 + i / TPR, j = i % TPR;
        const float2 *in = reinterpret_cast<const float2 *>(src + (long long)(CS * q + r) * a.rnxp);
        float2 *row = A + q * P;
        if (j == 0) {
          if (off) cp_async8(row + 1, in);
        } else {
          const int e = 2 * (j - 1) + off;  // first element of the pair
          cp_async16(row + off + e, in + e);
        }
      }
    } else {
      for (int i = tid; i < nr * NH; i += kPlaneThreads) {
        const int q = q0 + i / NH, e = i % NH;
        cp_async8(A + q * P + e, reinterpret_cast<const float2 *>(src + (long long)(CS * q + r) * a.rnxp) + e);
      }
    }
    cp_async_commit();
  }
  for (int rd = 0; rd < NRX; ++rd) {
    const int q = rd * RPR + tid / TX, t = tid % TX;
    const bool act = q < NQ;
    float2 *row = A + (act ? q : 0) * P;
    if (rd + 1 < NRX) cp_async_wait<1>();
    else cp_async_wait<0>();
    __syncthreads();  // this round's rows (every thread's copies) and the tables
    float2 v[EX];
    if (act) {
#pragma unroll
      for (int b = 0; b < EX / R0X; ++b)
#pragma unroll
        for (int qq = 0; qq < R0X; ++qq) v[b * R0X + qq] = row[off + rr::stage_in<NH, 0, EX, TX>(t, b, qq)];
    }
    auto ix = [](int e) { return C::physx(e); };
    SmemStages<NH, -1, EX, TX, 0, true, decltype(ix)>::run(v, row, twx, t, act, ix);
    // split X_k = E_k + W^k O_k in registers: position k = t + TX m pairs
    // with NH - k, which thread TX - t of the row holds at m' = EX - 1 - m
    // (thread 0: its own position EX - m), one warp shuffle per output
    static_assert(TX <= 32 && (32 % TX) == 0, "a row's threads lie in one warp");
    const int lane = threadIdx.x & 31;
    const int srcl = lane - t + (TX - t) % TX;
    float2 X[EX + 1];
#pragma unroll
    for (int m = 0; m < EX; ++m) {
      const float2 send = v[last_reg<EX, RLX>(EX - 1 - m)];
      float2 zm = make_float2(__shfl_sync(0xffffffffu, send.x, srcl), __shfl_sync(0xffffffffu, send.y, srcl));
      if (t == 0) zm = v[last_reg<EX, RLX>(m == 0 ? 0 : EX - m)];
      const float2 zk = v[last_reg<EX, RLX>(m)];
      zm.y = -zm.y;
      const float2 e = cscale(cadd(zk, zm), 0.5f);
      const float2 d = csub(zk, zm);
      const float2 o = make_float2(0.5f * d.y, -0.5f * d.x);
      X[m] = cscale(cadd(e, cmul(post[t + TX * m], o)), a.scale);
    }
    {
      // X_NH from Z_0 alone (thread 0)
      const float2 zk = v[last_reg<EX, RLX>(0)];
      float2 zm = zk;
      zm.y = -zm.y;
      const float2 e = cscale(cadd(zk, zm), 0.5f);
      const float2 d = csub(zk, zm);
      const float2 o = make_float2(0.5f * d.y, -0.5f * d.x);
      X[EX] = cscale(cadd(e, cmul(post[NH], o)), a.scale);
    }
    __syncwarp();  // the row's exchange reads are done before the plain layout overwrites them
    if (act) {
#pragma unroll
      for (int m = 0; m < EX; ++m) row[t + TX * m] = X[m];
      if (t == 0) row[NH] = X[EX];
    }
  }
  __syncthreads();

  // 2. y, local: NQ points along this CTA's rows for every column kx,
  //    then the twiddle W_NY^{r k1}; in place in A
  constexpr int CPR = kPlaneThreads / TQ;  // columns per round
  constexpr int NRQ = (CX + CPR - 1) / CPR;
  for (int rd = 0; rd < NRQ; ++rd) {
    const int kx = rd * CPR + tid % CPR, t = tid / CPR;
    const bool act = kx < CX;
    float2 v[EQ];
    if (act) {
#pragma unroll
      for (int b = 0; b < EQ / R0Q; ++b)
#pragma unroll
        for (int qq = 0; qq < R0Q; ++qq) v[b * R0Q + qq] = A[rr::stage_in<NQ, 0, EQ, TQ>(t, b, qq) * P + kx];
    }
    auto iy = [kx](int e) { return e * P + (kx < CX ? kx : 0); };
    SmemStages<NQ, -1, EQ, TQ, 0, false, decltype(iy)>::run(v, A, twq, t, act, iy);
    // the last stage's outputs go to the very slots its inputs came from
    // (the stride-TQ set of this thread), and a round owns its columns:
    // no barrier before the write-back or between rounds
    if (act) {
#pragma unroll
      for (int b = 0; b < EQ / RLQ; ++b)
#pragma unroll
        for (int qq = 0; qq < RLQ; ++qq) {
          const int k1 = rr::stage_in<NQ, SQ - 1, EQ, TQ>(t, b, qq);
          A[k1 * P + kx] = cmul(v[b * RLQ + qq], twr[k1]);
        }
    }
  }

  // 3. the radix-CS stage across the cluster: this CTA's k1 range, every
  //    column; the CS outputs are spectrum rows k1 + NQ k2
  cl.sync();
  const float2 *Ar[CS];
#pragma unroll
  for (int s = 0; s < CS; ++s) Ar[s] = cl.map_shared_rank(A, s);
  // two items per thread and step: the 2 CS loads from the partners'
  // shared memory are issued before either item's butterfly
  constexpr int NI = C::QK * CX;
  for (int i0 = tid; i0 < NI; i0 += 2 * kPlaneThreads) {
    const int i1 = i0 + kPlaneThreads;
    const bool two = i1 < NI;
    const int k1a = r * C::QK + i0 / CX, kxa = i0 % CX;
    const int k1b = r * C::QK + (two ? i1 : i0) / CX, kxb = (two ? i1 : i0) % CX;
    float2 va[CS], vb[CS];
#pragma unroll
    for (int s = 0; s < CS; ++s) {
      va[s] = Ar[s][k1a * P + kxa];
      vb[s] = Ar[s][k1b * P + kxb];
    }
    Dft<CS, -1>::run(va);
#pragma unroll
    for (int k2 = 0; k2 < CS; ++k2) dst[(long long)(k1a + NQ * k2) * CX + kxa] = va[k2];
    if (two) {
      Dft<CS, -1>::run(vb);
#pragma unroll
      for (int k2 = 0; k2 < CS; ++k2) dst[(long long)(k1b + NQ * k2) * CX + kxb] = vb[k2];
    }
  }
  cl.sync();  // partners are done reading this CTA's shared memory
}

// ------------------------------------------------------------------ inverse
template <int NH, int NY, int CS>
__global__ void __launch_bounds__(kPlaneThreads, kPlaneMinBlocks) k_plane_xy_inv(const __grid_constant__ PlaneArgs a) {
  using C = PlaneCfg<NH, NY, CS>;
  constexpr int NQ = C::NQ, CX = C::CX, P = C::P, EX = C::EX, TX = C::TX, EQ = C::EQ, TQ = C::TQ;
  constexpr int R0X = C::R0X, SX = CtRadix::count(NH), RLX = CtRadix::at(NH, SX - 1);
  constexpr int R0Q = CtRadix::at(NQ, 0), SQ = CtRadix::count(NQ), RLQ = CtRadix::at(NQ, SQ - 1);
  cg::cluster_group cl = cg::this_cluster();
  extern __shared__ float4 sm4[];
  float2 *twx = reinterpret_cast<float2 *>(sm4);
  float2 *post = twx + NH;
  float2 *twq = post + NH + 1;
  float2 *twr = twq + NQ;  // W_NY^{-r k1}
  float2 *A = twx + C::TABN + (C::TABN & 1);
  const int tid = threadIdx.x, r = (int)cl.block_rank();
  for (int i = tid; i < NH; i += kPlaneThreads) twx[i] = a.twx[i];
  for (int i = tid; i <= NH; i += kPlaneThreads) post[i] = a.post[i];
  for (int i = tid; i < NQ; i += kPlaneThreads) {
    twq[i] = a.twq[i];
    twr[i] = cconj(a.twy[(r * i) % NY]);
  }
  const int plane = blockIdx.x / CS;
  const long long pr = (long long)a.rnxp * a.nyp;
  const float2 *src = reinterpret_cast<const float2 *>(a.src + (long long)plane * pr);
  float *dst = a.dst + (long long)plane * pr;
  const float *add = a.add ? a.add + (long long)plane * pr : nullptr;

  // 1. the inverse radix-CS stage for this CTA's k1 range from HBM; value
  //    t goes to CTA t's shared memory (every partner is running and done
  //    with any earlier use of its buffer: cluster barrier first)
  cl.sync();
  float2 *At[CS];
#pragma unroll
  for (int s = 0; s < CS; ++s) At[s] = cl.map_shared_rank(A, s);
  // kInvItems items per thread and step: their kInvItems x CS loads from
  // HBM are in flight together (an item past the end reloads item i0 and
  // stores nothing)
  constexpr int NI = C::QK * CX;
  constexpr int IPS = kInvItems;
  for (int i0 = tid; i0 < NI; i0 += IPS * kPlaneThreads) {
    float2 v[IPS][CS];
    int k1[IPS], kx[IPS];
#pragma unroll
    for (int u = 0; u < IPS; ++u) {
      const int i = i0 + u * kPlaneThreads < NI ? i0 + u * kPlaneThreads : i0;
      k1[u] = r * C::QK + i / CX;
      kx[u] = i % CX;
#pragma unroll
      for (int k2 = 0; k2 < CS; ++k2) v[u][k2] = src[(long long)(k1[u] + NQ * k2) * CX + kx[u]];
    }
#pragma unroll
    for (int u = 0; u < IPS; ++u) {
      if (i0 + u * kPlaneThreads < NI) {
        Dft<CS, 1>::run(v[u]);
#pragma unroll
        for (int s = 0; s < CS; ++s) At[s][k1[u] * P + kx[u]] = v[u][s];
      }
    }
  }
  cl.sync();

  // 2. y, local: twiddle W_NY^{-r k1}, then the NQ-point inverse along k1
  //    for every column; outputs are rows p (y = CS p + r), in place
  constexpr int CPR = kPlaneThreads / TQ;
  constexpr int NRQ = (CX + CPR - 1) / CPR;
  for (int rd = 0; rd < NRQ; ++rd) {
    const int kx = rd * CPR + tid % CPR, t = tid / CPR;
    const bool act = kx < CX;
    float2 v[EQ];
    if (act) {
#pragma unroll
      for (int b = 0; b < EQ / R0Q; ++b)
#pragma unroll
        for (int qq = 0; qq < R0Q; ++qq) {
          const int k1 = rr::stage_in<NQ, 0, EQ, TQ>(t, b, qq);
          v[b * R0Q + qq] = cmul(A[k1 * P + kx], twr[k1]);
        }
    }
    auto iy = [kx](int e) { return e * P + (kx < CX ? kx : 0); };
    SmemStages<NQ, 1, EQ, TQ, 0, false, decltype(iy)>::run(v, A, twq, t, act, iy);
    // outputs to the slots of the last stage's inputs; rounds own their
    // columns (see the forward)
    if (act) {
#pragma unroll
      for (int b = 0; b < EQ / RLQ; ++b)
#pragma unroll
        for (int qq = 0; qq < RLQ; ++qq) A[rr::stage_in<NQ, SQ - 1, EQ, TQ>(t, b, qq) * P + kx] = v[b * RLQ + qq];
    }
  }
  __syncthreads();  // every column is done before the rows are read

  // 3. x C2R of every row to HBM (scale, addend, zero pad)
  constexpr int RPR = kPlaneThreads / TX;
  constexpr int NRX = (NQ + RPR - 1) / RPR;
  for (int rd = 0; rd < NRX; ++rd) {
    const int q = rd * RPR + tid / TX, t = tid % TX;
    const bool act = q < NQ;
    float2 *row = A + (act ? q : 0) * P;
    float2 v[EX];
    if (act) {
      // Z'[k] = (X_k + conj X_{NH-k}) + i W^{-k} (X_k - conj X_{NH-k}); the
      // imaginary parts of DC and Nyquist are ignored, as a C2R does
#pragma unroll
      for (int b = 0; b < EX / R0X; ++b)
#pragma unroll
        for (int qq = 0; qq < R0X; ++qq) {
          const int k = rr::stage_in<NH, 0, EX, TX>(t, b, qq);
          float2 x0 = row[k], x1 = row[NH - k];
          if (k == 0) { x0.y = 0.f; x1.y = 0.f; }
          x1.y = -x1.y;
          const float2 e = cadd(x0, x1);
          float2 w = post[k];
          w.y = -w.y;
          const float2 o = cmul(csub(x0, x1), w);
          v[b * R0X + qq] = make_float2(e.x - o.y, e.y + o.x);
        }
    }
    __syncwarp();  // the row's spectrum is read before the exchanges overwrite it (a row lies in one warp)
    auto ix = [](int e) { return C::physx(e); };
    SmemStages<NH, 1, EX, TX, 0, true, decltype(ix)>::run(v, row, twx, t, act, ix);
    if (act) {
      const long long ro = (long long)(CS * q + r) * a.rnxp;
      float2 *orow = reinterpret_cast<float2 *>(dst + ro);
      const float2 *arow = add ? reinterpret_cast<const float2 *>(add + ro) : nullptr;
#pragma unroll
      for (int b = 0; b < EX / RLX; ++b)
#pragma unroll
        for (int qq = 0; qq < RLX; ++qq) {
          const int m = rr::stage_in<NH, SX - 1, EX, TX>(t, b, qq);
          float2 x = cscale(v[b * RLX + qq], a.scale);
          if (arow) x = cadd(x, arow[m]);
          orow[m] = x;
        }
      if (t == 0) orow[NH] = make_float2(0.f, 0.f);
    }
    // the next round works on other rows: no barrier
  }
}

template <int NH, int NY, int CS>
int launch_plane(const PlaneArgs &a, int dir, cudaStream_t s) {
  using C = PlaneCfg<NH, NY, CS>;
  const void *fn = dir < 0 ? (const void *)k_plane_xy_fwd<NH, NY, CS> : (const void *)k_plane_xy_inv<NH, NY, CS>;
  int rc = func_smem(fn, C::smem);
  if (rc) return rc;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(a.nplanes * CS));
  cfg.blockDim = dim3(kPlaneThreads);
  cfg.dynamicSmemBytes = C::smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = CS;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (dir < 0) CRAVA_CUDA_TRY(cudaLaunchKernelEx(&cfg, k_plane_xy_fwd<NH, NY, CS>, a));
  else CRAVA_CUDA_TRY(cudaLaunchKernelEx(&cfg, k_plane_xy_inv<NH, NY, CS>, a));
  note_launch();
  return CRAVA_GPU_OK;
}

}  // namespace

bool plane_xy_supported(const Geom &g) {
  return (g.nxp == 256 && g.nyp == 256) || (g.nxp == 128 && g.nyp == 128);
}

int plane_xy_tables(const Geom &g, float2 **twq, float2 **twy) {
  *twq = *twy = nullptr;
  if (!plane_xy_supported(g)) return CRAVA_GPU_OK;
  const int ny = g.nyp, nq = g.nyp == 256 ? 64 : 64;
  std::vector<float2> q(nq), y(ny);
  for (int k = 0; k < nq; ++k) {
    const double ang = -2.0 * M_PI * (double)k / (double)nq;
    q[k] = make_float2((float)cos(ang), (float)sin(ang));
  }
  for (int k = 0; k < ny; ++k) {
    const double ang = -2.0 * M_PI * (double)k / (double)ny;
    y[k] = make_float2((float)cos(ang), (float)sin(ang));
  }
  CRAVA_CUDA_TRY(cudaMalloc(twq, sizeof(float2) * nq));
  CRAVA_CUDA_TRY(cudaMalloc(twy, sizeof(float2) * ny));
  CRAVA_CUDA_TRY(cudaMemcpy(*twq, q.data(), sizeof(float2) * nq, cudaMemcpyHostToDevice));
  CRAVA_CUDA_TRY(cudaMemcpy(*twy, y.data(), sizeof(float2) * ny, cudaMemcpyHostToDevice));
  return CRAVA_GPU_OK;
}

int plane_xy(const FftPlans &p, const float *src, float *dst, int dir, float scale, const float *addend,
             cudaStream_t s) {
  const Geom &g = p.g;
  if (!plane_xy_supported(g) || !p.twq || !p.twy) return CRAVA_GPU_ERR_ARG;
  PlaneArgs a{};
  a.src = src ? src : dst;
  a.dst = dst;
  a.add = addend;
  a.rnxp = g.rnxp;
  a.nyp = g.nyp;
  a.nplanes = g.nzp;
  a.scale = scale;
  a.twx = p.x.tw;
  a.post = p.xpost;
  a.twq = p.twq;
  a.twy = p.twy;
  if (g.nxp == 256 && g.nyp == 256) return launch_plane<128, 256, 4>(a, dir, s);
  return launch_plane<64, 128, 2>(a, dir, s);
}

}  // namespace crava
