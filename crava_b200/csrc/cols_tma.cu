// cols_tma.cu -- the z pass of the register-resident transform with its
// tiles brought into shared memory by the Tensor Memory Accelerator.
//
// The z pass transforms the cnxp * nyp lines of a grid along z, line f's
// element z at f + z L (L = cnxp nyp complex values per z plane).  Eight
// adjacent lines form a tile: a 64-byte run of every z plane, which one 2-D
// TMA box (16 floats x up to 256 planes) describes exactly, whatever the
// plane size, as long as a plane is a whole number of 16-byte units (L
// even) and the grid is 16-byte aligned.  (The y and x passes have no such
// box: a padded row is rnxp = 2 (nxp/2 + 1) floats, so every other row
// starts 8 bytes off a 16-byte boundary.)
//
// Each CTA is persistent over the tiles t = blockIdx.x + k gridDim.x and
// keeps two tile buffers: while it transforms tile k in one buffer, the TMA
// brings tile k + 1 into the other, so the HBM reads of the next tile run
// under the arithmetic of this one (the register-resident kernel of fft.cu
// waits for its loads with nothing else to do).  Within a tile the work is
// that kernel's: the stage-0 inputs go shared -> registers, every radix
// stage is the Stockham stage of fft_rr.cuh, the S - 1 exchanges reuse the
// tile's buffer, and the last stage writes HBM directly (16-byte stores of
// two adjacent lines).  Same radices, twiddles and butterflies, so the
// values equal the other z passes bit for bit.
//
// Shared rows are 64 bytes (8 lines); a warp phase covers the rows of two
// consecutive thread positions t, t + 1.  They must fall into different
// bank halves: the landed tile (natural row order) and every exchange read
// satisfy that, and the first stage's writes (rows j R_0 + q, j = t, t + 1)
// do once exchange row o is stored at o ^ ((o >> log2 R_0) & 1).
//
// Waits on the tile barriers are bounded: a CTA that gives up counts the
// event in g_tile_wait_timeouts (crava_gpu_get_stats), waits, again
// bounded, for the copies it still has in flight, and returns.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <stdlib.h>

#include "fft.cuh"
#include "fft_rr.cuh"

namespace crava {

__device__ unsigned long long g_tile_wait_timeouts;

namespace {

constexpr int kTileLines = 8;       // lines per tile (64 bytes of a z plane)
constexpr int kBoxRows = 256;       // the TMA box limit per dimension
constexpr uint32_t kWaitRounds = 1u << 22;

__host__ __device__ constexpr int ilog2c(int n) { return n <= 1 ? 0 : 1 + ilog2c(n / 2); }

template <int N>
struct ZT {
  static constexpr int E = rr::max_radix(N);
  static constexpr int T = N / E;
  static constexpr int CPT = E >= 16 ? 1 : 2;  // lines per thread
  static constexpr int NP = kTileLines / CPT;
  static constexpr int NTH = NP * T;
  // resident CTAs per SM the register budget is sized for (the shared
  // memory of two tile buffers allows as many)
  static constexpr int MINB = N == 512 ? 3 : N == 256 ? 6 : N == 128 ? 12 : 16;
  static constexpr int K0 = ilog2c(CtRadix::at(N, 0));
  static constexpr int BUF = N * kTileLines;  // float2 per tile buffer
  static constexpr int BOXROWS = N > kBoxRows ? kBoxRows : N;
  static constexpr int NBOX = N / BOXROWS;
  static constexpr uint32_t BYTES = (uint32_t)BUF * 8u;
  static __device__ __forceinline__ int phys(int o) { return o ^ ((o >> K0) & 1); }
  static constexpr size_t smem() { return 1024 + 2 * (size_t)BYTES + 8 * (size_t)rr::tw_slots<N>() + 16; }
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint32_t a, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(a), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t a, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(a), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t a, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n"
      ".reg .pred p;\n"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      "selp.u32 %0, 1, 0, p;\n"
      "}\n"
      : "=r"(done)
      : "r"(a), "r"(parity)
      : "memory");
  return done != 0;
}
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t a, uint32_t parity) {
  for (uint32_t i = 0; i < kWaitRounds; ++i)
    if (mbar_try_wait(a, parity)) return true;
  return false;
}
// Generic-proxy accesses of this thread to shared memory are ordered before
// later async-proxy (TMA) writes to it.
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap *tm, int x, int y, uint32_t mbar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(tm)), "r"(x), "r"(y), "r"(mbar)
      : "memory");
}

// Tile `tile` (lines tile*8 .. tile*8 + 7, all N planes) into the buffer at
// shared address dst; completion on the barrier at mbar.
template <int N>
__device__ __forceinline__ void issue_tile(const CUtensorMap *tm, uint32_t dst, uint32_t mbar, int tile) {
  using Z = ZT<N>;
  mbar_expect_tx(mbar, Z::BYTES);
#pragma unroll
  for (int b = 0; b < Z::NBOX; ++b)
    tma_load_2d(dst + (uint32_t)(b * Z::BOXROWS * kTileLines * 8), tm, tile * 2 * kTileLines, b * Z::BOXROWS, mbar);
}

struct ZTmaArgs {
  float2 *data;
  long long L;  // lines, = complex values per z plane
  int ntiles;
  int tpc;  // tiles per CTA (0: persistent grid of the resident CTAs)
  const float2 *tw;
  ZPrior zp;  // forward pass of a covariance grid: the band-gated rule (inv null: none)
};

template <int N, int DIR, int S>
struct ZTmaStages {
  using Z = ZT<N>;
  // v holds the inputs of stage S
  static __device__ __forceinline__ void run(float2 (&v)[Z::CPT][Z::E], float2 *B, const float2 *tw, int t, int p,
                                             float2 *g, long long L, bool ok, const ZPrior &zp, long long f,
                                             unsigned gmask) {
    constexpr int E = Z::E, T = Z::T, CPT = Z::CPT, R = CtRadix::at(N, S);
#pragma unroll
    for (int c = 0; c < CPT; ++c) rr::stage_compute_st<N, S, DIR, E, T>(v[c], tw, t);
    if constexpr (S + 1 == CtRadix::count(N)) {
      // last stage: the outputs sit at the positions loaded, straight to HBM
      if (DIR < 0 && gmask && ok) {
        // band-gated kz planes of a covariance grid (gmask: this thread's
        // output registers on them): the prior rule (the CPT lines of a
        // thread are f, f + 1: L is even)
#pragma unroll
        for (int b = 0; b < E / R; ++b)
#pragma unroll
          for (int q = 0; q < R; ++q) {
            if ((gmask >> (b * R + q)) & 1u) {
              const int e = rr::stage_in<N, S, E, T>(t, b, q);
#pragma unroll
              for (int c = 0; c < CPT; ++c)
                v[c][b * R + q] = zprior_apply(zp, v[c][b * R + q], f + c + (long long)e * L);
            }
          }
      }
      if (ok) {
#pragma unroll
        for (int b = 0; b < E / R; ++b)
#pragma unroll
          for (int q = 0; q < R; ++q) {
            const long long e = rr::stage_in<N, S, E, T>(t, b, q);
            if (CPT == 2)
              *reinterpret_cast<float4 *>(g + e * L) =
                  make_float4(v[0][b * R + q].x, v[0][b * R + q].y, v[CPT - 1][b * R + q].x, v[CPT - 1][b * R + q].y);
            else
              g[e * L] = v[0][b * R + q];
          }
      }
    } else {
      if (S > 0) __syncthreads();  // every thread has read this stage's inputs
#pragma unroll
      for (int b = 0; b < E / R; ++b)
#pragma unroll
        for (int q = 0; q < R; ++q) {
          const int o = Z::phys(rr::stage_out<N, S, T>(t, b, q));
          if (CPT == 2)
            *reinterpret_cast<float4 *>(B + o * kTileLines + 2 * p) =
                make_float4(v[0][b * R + q].x, v[0][b * R + q].y, v[CPT - 1][b * R + q].x, v[CPT - 1][b * R + q].y);
          else
            B[o * kTileLines + p] = v[0][b * R + q];
        }
      __syncthreads();
      constexpr int R2 = CtRadix::at(N, S + 1);
#pragma unroll
      for (int b = 0; b < E / R2; ++b)
#pragma unroll
        for (int q = 0; q < R2; ++q) {
          const int e = Z::phys(rr::stage_in<N, S + 1, E, T>(t, b, q));
          if (CPT == 2) {
            const float4 x = *reinterpret_cast<const float4 *>(B + e * kTileLines + 2 * p);
            v[0][b * R2 + q] = make_float2(x.x, x.y);
            v[CPT - 1][b * R2 + q] = make_float2(x.z, x.w);
          } else {
            v[0][b * R2 + q] = B[e * kTileLines + p];
          }
        }
      ZTmaStages<N, DIR, S + 1>::run(v, B, tw, t, p, g, L, ok, zp, f, gmask);
    }
  }
};

template <int N, int DIR>
__global__ void __launch_bounds__(ZT<N>::NTH, ZT<N>::MINB) k_cols_z_tma(const __grid_constant__ CUtensorMap tm,
                                                          const __grid_constant__ ZTmaArgs a) {
  using Z = ZT<N>;
  constexpr int E = Z::E, T = Z::T, CPT = Z::CPT, NP = Z::NP, R0 = CtRadix::at(N, 0);
  extern __shared__ unsigned char smraw[];
  // two tile buffers on a 1024-byte boundary, then the per-stage twiddle
  // tables and the two tile barriers
  const uint32_t s0 = smem_u32(smraw);
  const uint32_t pad = ((s0 + 1023u) & ~1023u) - s0;
  float2 *buf = reinterpret_cast<float2 *>(smraw + pad);
  float2 *tw = buf + 2 * Z::BUF;
  const uint32_t bufs = s0 + pad;
  const uint32_t mbs = smem_u32(tw + rr::tw_slots<N>());
  const int tid = threadIdx.x;
  const int p = tid % NP, t = tid / NP;
  if (tid == 0) {
    mbar_init(mbs, 1);
    mbar_init(mbs + 8, 1);
    mbar_init_fence();
  }
  rr::tw_stages_fill<N>(tw, a.tw, tid, Z::NTH);
  const unsigned gmask = DIR < 0 ? zprior_mask<N, E, T>(a.zp, t) : 0u;
  __syncthreads();
  // tiles of this CTA: blockIdx.x, + gridDim.x, ... (persistent grid,
  // tpc 0) or the run of tpc tiles from blockIdx.x * tpc
  const int G = a.tpc > 0 ? 1 : (int)gridDim.x;
  int tile = a.tpc > 0 ? (int)blockIdx.x * a.tpc : (int)blockIdx.x;
  const int end = a.tpc > 0 ? min(tile + a.tpc, a.ntiles) : a.ntiles;
  if (tid == 0) {
    if (tile < end) issue_tile<N>(&tm, bufs, mbs, tile);
    if (tile + G < end) issue_tile<N>(&tm, bufs + Z::BYTES, mbs + 8, tile + G);
  }
  int k = 0;
  bool gave_up = false;
  for (; tile < end; tile += G, ++k) {
    const int sb = k & 1;
    float2 *B = buf + sb * Z::BUF;
    const bool landed = mbar_wait_bounded(mbs + 8u * sb, (uint32_t)(k >> 1) & 1u);
    if (__syncthreads_or(!landed)) {
      gave_up = true;
      break;
    }
    float2 v[CPT][E];
#pragma unroll
    for (int b = 0; b < E / R0; ++b)
#pragma unroll
      for (int q = 0; q < R0; ++q) {
        const int e = rr::stage_in<N, 0, E, T>(t, b, q);
        if (CPT == 2) {
          const float4 x = *reinterpret_cast<const float4 *>(B + e * kTileLines + 2 * p);
          v[0][b * R0 + q] = make_float2(x.x, x.y);
          v[CPT - 1][b * R0 + q] = make_float2(x.z, x.w);
        } else {
          v[0][b * R0 + q] = B[e * kTileLines + p];
        }
      }
    __syncthreads();  // the landed tile is read before the first exchange overwrites it
    const long long f = (long long)tile * kTileLines + p * CPT;
    ZTmaStages<N, DIR, 0>::run(v, B, tw, t, p, a.data + f, a.L, f < a.L, a.zp, f, gmask);
    fence_proxy_async_smem();
    __syncthreads();  // every thread is done with this buffer
    if (tid == 0 && tile + 2 * G < end) issue_tile<N>(&tm, bufs + sb * Z::BYTES, mbs + 8u * sb, tile + 2 * G);
  }
  if (gave_up && tid == 0) {
    atomicAdd(&g_tile_wait_timeouts, 1ull);
    // the copies still in flight: this tile's and the next one's
    mbar_wait_bounded(mbs + 8u * (k & 1), (uint32_t)(k >> 1) & 1u);
    if (tile + G < end) mbar_wait_bounded(mbs + 8u * ((k + 1) & 1), (uint32_t)((k + 1) >> 1) & 1u);
  }
}

// Tiles per CTA: a run of a few tiles per CTA leaves the hardware to
// balance the CTAs (and lets kernels of other grids, on other streams,
// share the SMs), where a persistent grid fixes every CTA's share up
// front.  CRAVA_ZTMA_TPC overrides it for measurements (0: persistent).
int tiles_per_cta() {
  static const int v = [] {
    const char *e = getenv("CRAVA_ZTMA_TPC");
    const int x = e ? atoi(e) : 4;
    return x < 0 || x > 64 ? 4 : x;
  }();
  return v;
}

using EncodeTiled = PFN_cuTensorMapEncodeTiled_v12000;

EncodeTiled encode_tiled() {
  static const EncodeTiled fn = [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return (EncodeTiled) nullptr;
    return reinterpret_cast<EncodeTiled>(p);
  }();
  return fn;
}

// Persistent grid: the resident CTAs of the device.
int resident_ctas(const void *fn, int nth, size_t smem, int *out) {
  int dev = 0, sms = 0, per = 0;
  CRAVA_CUDA_TRY(cudaGetDevice(&dev));
  CRAVA_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  CRAVA_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, nth, smem));
  *out = (per > 0 ? per : 1) * sms;
  return CRAVA_GPU_OK;
}

template <int N, int DIR>
int launch_z_tma(const CUtensorMap &tm, const ZTmaArgs &a, cudaStream_t s) {
  using Z = ZT<N>;
  const void *fn = (const void *)k_cols_z_tma<N, DIR>;
  int rc;
  if ((rc = func_smem(fn, Z::smem()))) return rc;
  int ctas = 0;
  if ((rc = resident_ctas(fn, Z::NTH, Z::smem(), &ctas))) return rc;
  const int grid = a.tpc > 0 ? (a.ntiles + a.tpc - 1) / a.tpc : (a.ntiles < ctas ? a.ntiles : ctas);
  k_cols_z_tma<N, DIR><<<grid, Z::NTH, Z::smem(), s>>>(tm, a);
  CRAVA_LAUNCH_CHECK();
  return CRAVA_GPU_OK;
}

}  // namespace

bool cols_z_tma_supported(const Geom &g, const void *data) {
  const long long L = (long long)g.cnxp * g.nyp;
  return rr::supported(g.nzp) && L % 2 == 0 && (reinterpret_cast<uintptr_t>(data) % 16) == 0 &&
         (L + kTileLines - 1) / kTileLines < (1LL << 31) && encode_tiled() != nullptr;
}

int cols_z_tma(const FftPlans &p, float2 *grid, int dir, cudaStream_t s, const ZPrior *zp) {
  const Geom &g = p.g;
  if (!cols_z_tma_supported(g, grid)) return CRAVA_GPU_ERR_ARG;
  const long long L = (long long)g.cnxp * g.nyp;
  const int n = g.nzp;
  CUtensorMap tm;
  const cuuint64_t dims[2] = {(cuuint64_t)(2 * L), (cuuint64_t)n};
  const cuuint64_t strides[1] = {(cuuint64_t)L * 8};
  const cuuint32_t box[2] = {2 * kTileLines, (cuuint32_t)(n > kBoxRows ? kBoxRows : n)};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = encode_tiled()(&tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, grid, dims, strides, box, estr,
                                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return CRAVA_GPU_ERR_ARG;
  ZTmaArgs a;
  a.data = grid;
  a.L = L;
  a.ntiles = (int)((L + kTileLines - 1) / kTileLines);
  a.tpc = tiles_per_cta();
  a.tw = p.z.tw;
  if (zp && dir < 0) a.zp = *zp;
  switch (n) {
    case 64: return dir < 0 ? launch_z_tma<64, -1>(tm, a, s) : launch_z_tma<64, 1>(tm, a, s);
    case 128: return dir < 0 ? launch_z_tma<128, -1>(tm, a, s) : launch_z_tma<128, 1>(tm, a, s);
    case 256: return dir < 0 ? launch_z_tma<256, -1>(tm, a, s) : launch_z_tma<256, 1>(tm, a, s);
    case 512: return dir < 0 ? launch_z_tma<512, -1>(tm, a, s) : launch_z_tma<512, 1>(tm, a, s);
    default: return CRAVA_GPU_ERR_ARG;
  }
}

int tile_wait_timeouts(unsigned long long *out) {
  CRAVA_CUDA_TRY(cudaMemcpyFromSymbol(out, g_tile_wait_timeouts, sizeof *out));
  return CRAVA_GPU_OK;
}

}  // namespace crava
