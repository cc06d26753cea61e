// noalloc.cu -- crava_gpu_posterior_noalloc: the per-bin posterior solve
// (crava_gpu_posterior) for callers that cannot allocate device memory.
//
// Some callers own every byte of HBM through their own arena -- a
// framework's caching allocator or a pool reserved up front -- where a
// cudaMalloc either fails or breaks the owner's accounting, and some run in
// loops that cannot afford the device synchronisation a cudaMalloc/cudaFree
// may imply.  The regular entry points allocate in crava_gpu_create (plans,
// per-kz tables, counters).  This entry point needs no context and
// allocates nothing: the solve's scratch -- the staged wavelets, the per-kz
// operator tables and the failure counters -- lives in one file-scope
// __device__ array of fixed size (kScratchBytes), which every GPU that
// loads the library holds until the process exits.  The caller passes the
// parameters (host) and the transformed grids (device), as for
// crava_gpu_posterior.
//
// Set-up: the first call on a device, with that device current, resolves
// the array's device address with cudaGetSymbolAddress and caches it for
// that device.  Make that first call before any stream capture.  The cached
// address belongs to the device's current primary context: after
// cudaDeviceReset (or anything else that destroys and re-creates the
// primary context) the array is re-created elsewhere and the cached address
// is stale: a process that resets a device must not call this entry point
// on that device again.
// Sharing: every call on a device uses the same array and the array keeps
// the last call's contents; each call rewrites the tables and clears the
// counters before use.  Calls whose work overlaps on the GPU (different
// streams, or different host threads on the same device) race on the
// array: serialise them.
#include <cstring>
#include <mutex>
#include <vector>

#include "common.cuh"
#include "solve.cuh"

namespace crava {
namespace {

// Limits of the static scratch: nzp * ntheta <= 16384 (e.g. nzp 2048 with 8
// angles, nzp 4096 with 4) and nzp <= 4096.
constexpr size_t kMaxKzTheta = 16384;
constexpr size_t kMaxNzp = 4096;
constexpr size_t kAlign = 256;

constexpr size_t align_up(size_t n) { return (n + kAlign - 1) / kAlign * kAlign; }

// Layout: counters | wavelet [nt][nzp] | norms [nt] | wd | e1 | e2 | e3 | inv
constexpr size_t kOffCounters = 0;
constexpr size_t kOffWavelet = align_up(sizeof(DevCounters));
constexpr size_t kOffNorm = kOffWavelet + align_up(kMaxKzTheta * sizeof(float));
constexpr size_t kOffWd = kOffNorm + align_up(CRAVA_GPU_MAX_THETA * sizeof(float));
constexpr size_t kOffE1 = kOffWd + align_up(kMaxKzTheta * sizeof(float2));
constexpr size_t kOffE2 = kOffE1 + align_up(kMaxKzTheta * sizeof(float2));
constexpr size_t kOffE3 = kOffE2 + align_up(kMaxKzTheta * sizeof(float2));
constexpr size_t kOffInv = kOffE3 + align_up(kMaxKzTheta * sizeof(float));
constexpr size_t kScratchBytes = kOffInv + align_up(kMaxNzp * sizeof(int));  // ~0.5 MB

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
unsigned char *g_ptr[kMaxDevices] = {};

// Device address of g_scratch on the current device (set-up once per device).
int scratch_address(int dev, unsigned char **out) {
  if (dev < 0 || dev >= kMaxDevices) return CRAVA_GPU_ERR_ARG;
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!g_ptr[dev]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
    if (e != cudaSuccess) {
      set_last_error(e, "cudaGetSymbolAddress(scratch)", __FILE__, __LINE__);
      return CRAVA_GPU_ERR_CUDA;
    }
    g_ptr[dev] = static_cast<unsigned char *>(p);
  }
  *out = g_ptr[dev];
  return CRAVA_GPU_OK;
}

bool smooth_2357(int n) {
  if (n < 1) return false;
  for (int q : {2, 3, 5, 7})
    while (n % q == 0) n /= q;
  return n == 1;
}

}  // namespace
}  // namespace crava

using namespace crava;

extern "C" int crava_gpu_posterior_noalloc(const crava_gpu_params *p, const crava_gpu_grids *g,
                                           int precision, void *stream, crava_gpu_stats *stats) {
  if (!p || !g || !p->wavelet || !p->A || !p->theta_cov || !p->var0) return CRAVA_GPU_ERR_ARG;
  if (p->nxp < 2 || p->nyp < 1 || p->nzp < 2 || !smooth_2357(p->nzp)) return CRAVA_GPU_ERR_ARG;
  // the bounds of crava_gpu_create: they also keep the solve's grid of
  // ceil((nxp/2+1) nyp / 256) * nzp blocks below 2^31
  if (p->nxp > 8192 || p->nyp > 4096) return CRAVA_GPU_ERR_ARG;
  if (p->ntheta < 1 || p->ntheta > CRAVA_GPU_MAX_THETA || p->nz < 1 || !(p->lz > 0.0)) return CRAVA_GPU_ERR_ARG;
  if (precision < CRAVA_SOLVE_FP64 || precision > CRAVA_SOLVE_FP32) return CRAVA_GPU_ERR_ARG;
  if (p->thickness_mode != 0 && p->thickness_mode != 1) return CRAVA_GPU_ERR_ARG;
  if ((size_t)p->nzp > kMaxNzp || (size_t)p->nzp * p->ntheta > kMaxKzTheta) return CRAVA_GPU_ERR_TOO_LARGE;
  auto mis = [](const void *q) { return !q || (reinterpret_cast<uintptr_t>(q) & 7u) != 0; };
  for (int q = 0; q < 3; ++q) if (mis(g->mu[q])) return CRAVA_GPU_ERR_ARG;
  for (int l = 0; l < p->ntheta; ++l) if (mis(g->data[l])) return CRAVA_GPU_ERR_ARG;
  for (int t = 0; t < 6; ++t) if (mis(g->cov[t])) return CRAVA_GPU_ERR_ARG;
  if (mis(g->err_corr)) return CRAVA_GPU_ERR_ARG;

  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return CRAVA_GPU_ERR_NODEV;
  unsigned char *base = nullptr;
  int rc = scratch_address(dev, &base);
  if (rc) return rc;
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int nt = p->ntheta, nzp = p->nzp;

  DevCounters *counters = reinterpret_cast<DevCounters *>(base + kOffCounters);
  float *d_wav = reinterpret_cast<float *>(base + kOffWavelet);
  float *d_norm = reinterpret_cast<float *>(base + kOffNorm);
  KzTables t;
  t.wd = reinterpret_cast<float2 *>(base + kOffWd);
  t.e1 = reinterpret_cast<float2 *>(base + kOffE1);
  t.e2 = reinterpret_cast<float2 *>(base + kOffE2);
  t.e3 = reinterpret_cast<float *>(base + kOffE3);
  t.inv = reinterpret_cast<int *>(base + kOffInv);

  // The scratch keeps the last call's contents: clear the counters and
  // rewrite every table entry this call reads.
  CRAVA_CUDA_TRY(cudaMemsetAsync(counters, 0, sizeof(DevCounters), s));
  CRAVA_CUDA_TRY(cudaMemcpyAsync(d_wav, p->wavelet, sizeof(float) * nzp * nt, cudaMemcpyHostToDevice, s));
  if (p->wavelet_norm)
    CRAVA_CUDA_TRY(cudaMemcpyAsync(d_norm, p->wavelet_norm, sizeof(float) * nt, cudaMemcpyHostToDevice, s));
  if ((rc = kz_tables_build_device(*p, d_wav, p->wavelet_norm ? d_norm : nullptr, &t, s))) return rc;

  SolveConsts c{};
  c.nt = nt;
  c.wnc = p->wnc;
  c.kappa_refine = kKappaRefineDefault;
  c.solve_shape = -1;
  for (int l = 0; l < nt; ++l) {
    for (int q = 0; q < 3; ++q) c.A[l][q] = p->A[3 * l + q];
    for (int m = 0; m < nt; ++m) c.theta[l][m] = p->theta_cov[l * nt + m];
  }
  const double *v = p->var0;
  c.var0[0] = v[0]; c.var0[1] = v[4]; c.var0[2] = v[8];
  c.var0[3] = v[1]; c.var0[4] = v[2]; c.var0[5] = v[5];
  SolveGrids sg{};
  for (int q = 0; q < 3; ++q) sg.mu[q] = reinterpret_cast<float2 *>(g->mu[q]);
  for (int l = 0; l < nt; ++l) sg.data[l] = reinterpret_cast<float2 *>(g->data[l]);
  for (int k = 0; k < 6; ++k) sg.cov[k] = reinterpret_cast<float2 *>(g->cov[k]);
  sg.err = reinterpret_cast<const float2 *>(g->err_corr);
  const long long cnxp = p->nxp / 2 + 1;
  if ((rc = posterior_solve(c, t, sg, cnxp * p->nyp * nzp, cnxp * p->nyp, precision, counters, s))) return rc;

  if (stats) {
    DevCounters h{};
    CRAVA_CUDA_TRY(cudaMemcpyAsync(&h, counters, sizeof h, cudaMemcpyDeviceToHost, s));
    CRAVA_CUDA_TRY(cudaStreamSynchronize(s));
    std::memset(stats, 0, sizeof *stats);
    stats->chol_fail_bins = (long long)h.chol_fail;
    stats->nonfinite_bins = (long long)h.nonfinite;
    stats->refined_bins = (long long)h.refined;
  }
  return CRAVA_GPU_OK;
}
