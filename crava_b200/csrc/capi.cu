// capi.cu -- the C ABI (include/crava_gpu.h): contexts, argument checks,
// stream ordering, statistics and the host-buffer entry point.
#include <atomic>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include <math.h>

#include "context.cuh"

namespace crava {

static std::atomic<long long> g_launches{0};
void note_launch(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
long long launches() { return g_launches.load(std::memory_order_relaxed); }

static thread_local std::string g_last_error;
void set_last_error(cudaError_t e, const char *what, const char *file, int line) {
  char buf[512];
  std::snprintf(buf, sizeof buf, "%s: %s (%s:%d)", what, cudaGetErrorString(e), file, line);
  g_last_error = buf;
}

static std::mutex g_smem_mu;
static std::vector<std::pair<std::pair<int, const void *>, size_t>> g_smem;

int func_smem(const void *fn, size_t bytes) {
  int dev = 0;
  CRAVA_CUDA_TRY(cudaGetDevice(&dev));
  static int dev_max = -1;
  std::lock_guard<std::mutex> lock(g_smem_mu);
  if (dev_max < 0) CRAVA_CUDA_TRY(cudaDeviceGetAttribute(&dev_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  if ((long long)bytes > dev_max) return CRAVA_GPU_ERR_ARG;
  if (bytes <= 48 * 1024) return CRAVA_GPU_OK;
  for (auto &e : g_smem)
    if (e.first.first == dev && e.first.second == fn) {
      if (e.second >= bytes) return CRAVA_GPU_OK;
      CRAVA_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
      e.second = bytes;
      return CRAVA_GPU_OK;
    }
  CRAVA_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  g_smem.push_back({{dev, fn}, bytes});
  return CRAVA_GPU_OK;
}

}  // namespace crava

using namespace crava;

namespace crava {

int check_ctx(const crava_gpu_ctx *c) { return c ? CRAVA_GPU_OK : CRAVA_GPU_ERR_ARG; }

bool smooth_2357(int n) {
  if (n < 1) return false;
  for (int p : {2, 3, 5, 7})
    while (n % p == 0) n /= p;
  return n == 1;
}

int validate(const crava_gpu_params *p) {
  if (!p) return CRAVA_GPU_ERR_ARG;
  if (p->nxp < 2 || p->nyp < 1 || p->nzp < 2) return CRAVA_GPU_ERR_ARG;
  if (!smooth_2357(p->nxp) || !smooth_2357(p->nyp) || !smooth_2357(p->nzp)) return CRAVA_GPU_ERR_ARG;
  // line lengths held in shared memory by the transform kernels
  if (p->nxp > 8192 || p->nyp > 4096 || p->nzp > 4096) return CRAVA_GPU_ERR_ARG;
  if (p->ntheta < 1 || p->ntheta > CRAVA_GPU_MAX_THETA) return CRAVA_GPU_ERR_ARG;
  if (!p->wavelet || !p->A || !p->theta_cov || !p->var0) return CRAVA_GPU_ERR_ARG;
  if (p->nz < 1 || !(p->lz > 0.0)) return CRAVA_GPU_ERR_ARG;
  if (p->precision < CRAVA_SOLVE_FP64 || p->precision > CRAVA_SOLVE_FP32) return CRAVA_GPU_ERR_ARG;
  if (p->thickness_mode != 0 && p->thickness_mode != 1) return CRAVA_GPU_ERR_ARG;
  return CRAVA_GPU_OK;
}

SolveGrids to_solve_grids(const crava_gpu_grids *gr, int nt) {
  SolveGrids s{};
  for (int q = 0; q < 3; ++q) s.mu[q] = reinterpret_cast<float2 *>(gr->mu[q]);
  for (int l = 0; l < nt; ++l) s.data[l] = reinterpret_cast<float2 *>(gr->data[l]);
  for (int t = 0; t < 6; ++t) s.cov[t] = reinterpret_cast<float2 *>(gr->cov[t]);
  s.err = reinterpret_cast<const float2 *>(gr->err_corr);
  return s;
}

int check_grids(const crava_gpu_ctx *c, const crava_gpu_grids *gr) {
  if (!gr) return CRAVA_GPU_ERR_ARG;
  for (int q = 0; q < 3; ++q) if (!gr->mu[q]) return CRAVA_GPU_ERR_ARG;
  for (int l = 0; l < c->p.ntheta; ++l) if (!gr->data[l]) return CRAVA_GPU_ERR_ARG;
  for (int t = 0; t < 6; ++t) if (!gr->cov[t]) return CRAVA_GPU_ERR_ARG;
  if (!gr->err_corr) return CRAVA_GPU_ERR_ARG;
  // float2 access needs 8-byte alignment
  auto mis = [](const void *ptr) { return (reinterpret_cast<uintptr_t>(ptr) & 7u) != 0; };
  for (int q = 0; q < 3; ++q) if (mis(gr->mu[q])) return CRAVA_GPU_ERR_ARG;
  for (int l = 0; l < c->p.ntheta; ++l) if (mis(gr->data[l])) return CRAVA_GPU_ERR_ARG;
  for (int t = 0; t < 6; ++t) if (mis(gr->cov[t])) return CRAVA_GPU_ERR_ARG;
  if (mis(gr->err_corr)) return CRAVA_GPU_ERR_ARG;
  return CRAVA_GPU_OK;
}

enum ProfKind {
  K_ROWS_FWD, K_COLS_Y_FWD, K_COLS_Z_FWD, K_SOLVE, K_COLS_Z_INV, K_COLS_Y_INV, K_ROWS_INV,
  K_SIM, K_PLANE_FWD, K_ZSOLVE, K_PLANE_INV, K_XY_FWD, K_XY_INV, K_NKINDS
};
const char *kKindName[K_NKINDS] = {"fft_rows_r2c", "fft_cols_y_fwd", "fft_cols_z_fwd", "posterior_solve",
                                   "fft_cols_z_inv", "fft_cols_y_inv", "fft_rows_c2r", "sim_noise_filter",
                                   "unit_plane_fwd", "unit_zsolve", "unit_plane_inv", "fft_xy_fwd", "fft_xy_inv"};

cudaEvent_t pool_get(crava_gpu_ctx *c) {
  if (!c->pool.empty()) { cudaEvent_t e = c->pool.back(); c->pool.pop_back(); return e; }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

// Records an event pair around one launch when profiling is on.
struct Scope {
  crava_gpu_ctx *c;
  int kind;
  double bytes;
  cudaEvent_t a = nullptr;
  // bytes: algorithmic traffic of the launch (default: per kind, see get_profile)
  Scope(crava_gpu_ctx *ctx, int k, double b = -1.0) : c(ctx), kind(k), bytes(b) {
    if (c->prof) { a = pool_get(c); cudaEventRecord(a, c->stream); }
  }
  ~Scope() {
    if (c->prof && a) {
      cudaEvent_t b = pool_get(c);
      cudaEventRecord(b, c->stream);
      c->recs.push_back({kind, a, b, bytes});
    }
  }
};

void prof_collect(crava_gpu_ctx *c) {
  for (auto &r : c->recs) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, r.a, r.b) == cudaSuccess) {
      const double G = (double)c->g.csize * 8.0;  // bytes of one grid
      const int nt = c->p.ntheta;
      double bytes = r.bytes >= 0 ? r.bytes
                   : r.kind == K_SOLVE ? (double)(19 + 2 * nt) * G
                   : r.kind == K_SIM   ? 9.0 * G
                                       : 2.0 * G;
      c->prof_ms[r.kind] += ms;
      c->prof_bytes[r.kind] += bytes;
      c->prof_n[r.kind] += 1;
    }
    c->pool.push_back(r.a);
    c->pool.push_back(r.b);
  }
  c->recs.clear();
}

int pass_forward(crava_gpu_ctx *c, const float *src, float *dst, int type, const ZPrior *zp) {
  int rc;
  if (use_plane_xy(c->plans)) {
    { Scope sc(c, K_XY_FWD); if ((rc = plane_xy(c->plans, src, dst, -1, forward_scale(c->g, type), nullptr, c->stream))) return rc; }
    { Scope sc(c, K_COLS_Z_FWD); if ((rc = fft_cols_z(c->plans, reinterpret_cast<float2 *>(dst), -1, c->stream, zp))) return rc; }
    return CRAVA_GPU_OK;
  }
  { Scope sc(c, K_ROWS_FWD); if ((rc = fft_rows(c->plans, dst, -1, forward_scale(c->g, type), c->stream, nullptr, src))) return rc; }
  { Scope sc(c, K_COLS_Y_FWD); if ((rc = fft_cols_y(c->plans, reinterpret_cast<float2 *>(dst), -1, c->stream))) return rc; }
  { Scope sc(c, K_COLS_Z_FWD); if ((rc = fft_cols_z(c->plans, reinterpret_cast<float2 *>(dst), -1, c->stream, zp))) return rc; }
  return CRAVA_GPU_OK;
}

int gated_prior_setup(crava_gpu_ctx *c, int precision, ZPrior zp[6], bool *on) {
  // (the flags are allocated with the context where the z pass has the
  // rule; a tuning that selects another z pass turns the rule off)
  *on = (precision == CRAVA_SOLVE_FP64 || precision == CRAVA_SOLVE_MIXED) && z_prior_supported(c->plans) &&
        c->tables.n_inv >= 0 && c->tables.order_inv && c->gated_nf;
  if (!*on) return CRAVA_GPU_OK;
  for (int t = 0; t < 6; ++t) {
    zp[t] = ZPrior{};
    zp[t].inv = c->tables.inv;
    zp[t].v = c->consts.var0[t];  // (0,0) (1,1) (2,2) (0,1) (0,2) (1,2): the cov grid order
    // FP64 form: sign(S0) |c| equals the rounded double rule while |S0|
    // keeps c / S0 and its product with S0 normal (fft.cuh); else the
    // double expression for every value
    const double av = fabs(zp[t].v);
    const bool exact = av == 0.0 || (av >= 1e-200 && av <= 1e200);
    zp[t].mode = precision == CRAVA_SOLVE_FP64 ? (exact ? 1 : 3) : 2;
    zp[t].nf_bits = c->gated_nf;
    zp[t].nf_any = c->gated_nf + c->gated_nf_words;
  }
  return CRAVA_GPU_OK;
}

int gated_prior_count(crava_gpu_ctx *c) {
  return gated_nonfinite_count(c->gated_nf, c->gated_nf_words, c->gated_nf + c->gated_nf_words, c->counters,
                               c->stream);
}

int pass_inverse(crava_gpu_ctx *c, float *grid, int type, const float *addend) {
  int rc;
  { Scope sc(c, K_COLS_Z_INV); if ((rc = fft_cols_z(c->plans, reinterpret_cast<float2 *>(grid), 1, c->stream))) return rc; }
  if (use_plane_xy(c->plans)) {
    Scope sc(c, K_XY_INV);
    return plane_xy(c->plans, grid, grid, 1, inverse_scale(c->g, type), addend, c->stream);
  }
  { Scope sc(c, K_COLS_Y_INV); if ((rc = fft_cols_y(c->plans, reinterpret_cast<float2 *>(grid), 1, c->stream))) return rc; }
  { Scope sc(c, K_ROWS_INV); if ((rc = fft_rows(c->plans, grid, 1, inverse_scale(c->g, type), c->stream, addend))) return rc; }
  return CRAVA_GPU_OK;
}

int pass_solve(crava_gpu_ctx *c, const crava_gpu_grids *gr, int precision, bool gated_done) {
  // bytes the in-place solve moves: (10+nt) spectra read and (9+nt)
  // written for an inverted bin, the six covariance spectra both ways for
  // a band-gated one unless the forward z passes did those (the FP32
  // reference-order kernel moves all of them)
  const double plane_bytes = (double)c->g.cnxp * c->g.nyp * 8.0;
  const int nt = c->p.ntheta, nzp = c->p.nzp;
  const double gated = gated_done ? 0.0 : 12.0 * (nzp - c->n_inverted);
  const double bytes = precision == CRAVA_SOLVE_FP32
                           ? (double)(19 + 2 * nt) * nzp * plane_bytes
                           : ((double)(19 + 2 * nt) * c->n_inverted + gated) * plane_bytes;
  Scope sc(c, K_SOLVE, bytes);
  SolveGrids sg = to_solve_grids(gr, c->p.ntheta);
  return posterior_solve(c->consts, c->tables, sg, c->g.csize, (long long)c->g.cnxp * c->g.nyp,
                         precision, c->counters, c->stream, gated_done);
}

int valid_precision(int prec) {
  return prec >= CRAVA_SOLVE_FP64 && prec <= CRAVA_SOLVE_FP32;
}

int ensure_workspace(crava_gpu_ctx *c) {
  if (c->W) return CRAVA_GPU_OK;
  const size_t n = (size_t)(10 + c->p.ntheta) * (size_t)c->uplan.wgrid;
  if (cudaMalloc(&c->W, n * sizeof(float2)) != cudaSuccess) { c->W = nullptr; return CRAVA_GPU_ERR_ALLOC; }
  return CRAVA_GPU_OK;
}

bool use_fused(const crava_gpu_ctx *c, int precision) {
  return c->fused && c->uplan.ok && precision != CRAVA_SOLVE_FP32;
}

// Grids of a crava_gpu_grids in unit order (mu 3, data nt, cov 6, err) with
// their FFTGrid types.
int unit_order(const crava_gpu_ctx *c, const crava_gpu_grids *g, float **ptr, int *type) {
  int i = 0;
  for (int q = 0; q < 3; ++q) { ptr[i] = g->mu[q]; type[i++] = CRAVA_GRID_PARAMETER; }
  for (int l = 0; l < c->p.ntheta; ++l) { ptr[i] = g->data[l]; type[i++] = CRAVA_GRID_DATA; }
  for (int t = 0; t < 6; ++t) { ptr[i] = g->cov[t]; type[i++] = CRAVA_GRID_COVARIANCE; }
  ptr[i] = g->err_corr; type[i++] = CRAVA_GRID_COVARIANCE;
  return i;
}

// Runs `n` independent per-grid steps, step i on lane i % lanes: the lane
// streams are forked from the context's stream and joined back to it, so
// kernels of different grids (e.g. an ALU-bound x pass and a shared-memory
// bound z pass) share the SMs.
template <typename F>
int on_lanes(crava_gpu_ctx *c, int n, F step) {
  const int L = c->lanes > 1 && c->lane_s[0]
                    ? (c->lanes > crava_gpu_ctx::kMaxLanes ? crava_gpu_ctx::kMaxLanes : c->lanes)
                    : 1;
  if (L == 1) {
    for (int i = 0; i < n; ++i) {
      int rc = step(i);
      if (rc) return rc;
    }
    return CRAVA_GPU_OK;
  }
  const cudaStream_t s0 = c->stream;
  CRAVA_CUDA_TRY(cudaEventRecord(c->lane_fork, s0));
  for (int k = 0; k < L; ++k) CRAVA_CUDA_TRY(cudaStreamWaitEvent(c->lane_s[k], c->lane_fork, 0));
  int rc = CRAVA_GPU_OK;
  for (int i = 0; i < n && !rc; ++i) {
    c->stream = c->lane_s[i % L];
    rc = step(i);
  }
  c->stream = s0;
  for (int k = 0; k < L; ++k) {
    CRAVA_CUDA_TRY(cudaEventRecord(c->lane_join[k], c->lane_s[k]));
    CRAVA_CUDA_TRY(cudaStreamWaitEvent(s0, c->lane_join[k], 0));
  }
  return rc;
}

int stage_event(crava_gpu_ctx *c, int i) {
  if (!c->capture) CRAVA_CUDA_TRY(cudaEventRecord(c->ev[i], c->stream));
  return CRAVA_GPU_OK;
}

int inverse_realisations(crava_gpu_ctx *c, float *const *grids, int n, const float *const post_mean[3]) {
  return on_lanes(c, n, [&](int k) { return pass_inverse(c, grids[k], CRAVA_GRID_PARAMETER, post_mean[k % 3]); });
}

int simulate_batches(crava_gpu_ctx *c, const float2 *const cv[6], const float *const post_mean[3],
                     uint64_t seed, uint64_t first, int count, float *const *out,
                     const unsigned long long *epoch, unsigned long long epoch_stride) {
  int rc;
  // batches of up to 8 realisations share one read and one factorisation
  // of the posterior covariance spectra per bin
  for (int r0 = 0; r0 < count; r0 += 8) {
    const int nr = count - r0 < 8 ? count - r0 : 8;
    float2 *o[24];
    for (int k = 0; k < 3 * nr; ++k) o[k] = reinterpret_cast<float2 *>(out[3 * r0 + k]);
    const uint64_t stream0 = 3ull * (first + (uint64_t)r0);
    {
      Scope sc(c, K_SIM, (6.0 + 3.0 * nr) * (double)c->g.csize * 8.0);
      if ((rc = noise_filter_multi(c->g, cv, o, nr, seed, stream0, epoch, 3ull * epoch_stride,
                                   c->counters, c->stream)))
        return rc;
    }
    if ((rc = on_lanes(c, 3 * nr, [&](int k) {
           return pass_inverse(c, out[3 * r0 + k], CRAVA_GRID_PARAMETER, post_mean[k % 3]);
         })))
      return rc;
  }
  return CRAVA_GPU_OK;
}

// Fused unit: plane forward (all grids, one launch), z transform + solve +
// inverse z (one launch), plane inverse (outputs, one launch).  The noise
// correlation output is not written (its transform stays in the workspace).
int run_unit_fused(crava_gpu_ctx *c, const crava_gpu_grids *in, const crava_gpu_grids *out,
                   int precision) {
  const cudaStream_t s = c->stream;
  int rc;
  if ((rc = ensure_workspace(c))) return rc;
  float *src[kMaxUnitGrids], *dst[kMaxUnitGrids];
  int type[kMaxUnitGrids];
  const int G = unit_order(c, in, src, type);
  unit_order(c, out, dst, type);
  float2 *w[kMaxUnitGrids];
  float fs[kMaxUnitGrids], is[kMaxUnitGrids];
  for (int i = 0; i < G; ++i) {
    w[i] = c->W + (size_t)i * c->uplan.wgrid;
    fs[i] = forward_scale(c->g, type[i]);
    is[i] = inverse_scale(c->g, type[i]);
  }
  const double gb = (double)c->g.csize * 8.0;
  const double wb = (double)c->uplan.wgrid * 8.0;
  CRAVA_CUDA_TRY(cudaMemsetAsync(c->counters, 0, sizeof(DevCounters), s));
  if ((rc = stage_event(c, 0))) return rc;
  {
    Scope sc(c, K_PLANE_FWD, G * (gb + wb));
    if ((rc = unit_plane_forward(c->uplan, c->plans, src, w, fs, G, s))) return rc;
  }
  if ((rc = stage_event(c, 1))) return rc;
  {
    Scope sc(c, K_ZSOLVE, (2 * G - 1) * wb);
    if ((rc = unit_zsolve(c->uplan, c->plans, c->consts, c->tables, w, precision, c->counters, s))) return rc;
  }
  if ((rc = stage_event(c, 2))) return rc;
  {
    Scope sc(c, K_PLANE_INV, (G - 1) * (gb + wb));
    if ((rc = unit_plane_inverse(c->uplan, c->plans, w, dst, is, nullptr, G - 1, s))) return rc;
  }
  if ((rc = stage_event(c, 3))) return rc;
  c->timed = !c->capture;
  return CRAVA_GPU_OK;
}

// The posterior unit reading the real inputs from `in` and leaving the
// outputs in `out` (in == out is the reference's in-place behaviour).
int run_unit(crava_gpu_ctx *c, const crava_gpu_grids *in, const crava_gpu_grids *out,
             int precision) {
  if (use_fused(c, precision)) return run_unit_fused(c, in, out, precision);
  const cudaStream_t s = c->stream;
  int rc;
  CRAVA_CUDA_TRY(cudaMemsetAsync(c->counters, 0, sizeof(DevCounters), s));
  if ((rc = stage_event(c, 0))) return rc;
  float *src[kMaxUnitGrids], *dst[kMaxUnitGrids];
  int type[kMaxUnitGrids];
  const int G = unit_order(c, in, src, type);
  unit_order(c, out, dst, type);
  // the band-gated bins of the six covariance grids: done by their forward
  // z passes where the plans allow it, and the solve visits the inverted
  // planes only
  ZPrior zp[6];
  bool gated = false;
  if ((rc = gated_prior_setup(c, precision, zp, &gated))) return rc;
  const int c0 = 3 + c->p.ntheta;  // first covariance grid in unit order
  if ((rc = on_lanes(c, G, [&](int i) {
         const ZPrior *z = gated && i >= c0 && i < c0 + 6 ? &zp[i - c0] : nullptr;
         return pass_forward(c, src[i], dst[i], type[i], z);
       })))
    return rc;
  if (gated && (rc = gated_prior_count(c))) return rc;
  if ((rc = stage_event(c, 1))) return rc;
  if ((rc = pass_solve(c, out, precision, gated))) return rc;
  if ((rc = stage_event(c, 2))) return rc;
  // the noise correlation (last in unit order) is not an output
  if ((rc = on_lanes(c, G - 1, [&](int i) { return pass_inverse(c, dst[i], type[i]); }))) return rc;
  if ((rc = stage_event(c, 3))) return rc;
  c->timed = !c->capture;
  return CRAVA_GPU_OK;
}

}  // namespace crava

extern "C" {

const char *crava_gpu_status_string(int status) {
  switch (status) {
    case CRAVA_GPU_OK: return "ok";
    case CRAVA_GPU_ERR_ARG: return "invalid argument";
    case CRAVA_GPU_ERR_ALLOC: return "allocation failed";
    case CRAVA_GPU_ERR_CUDA: return g_last_error.empty() ? "CUDA error" : g_last_error.c_str();
    case CRAVA_GPU_ERR_TIMEOUT: return "device wait timed out";
    case CRAVA_GPU_ERR_STATE: return "call out of order";
    case CRAVA_GPU_ERR_NODEV: return "no CUDA device";
    case CRAVA_GPU_ERR_TOO_LARGE:
      return "size exceeds the static scratch of crava_gpu_posterior_noalloc "
             "(nzp <= 4096, nzp * ntheta <= 16384)";
    default: return "unknown status";
  }
}

long long crava_gpu_launch_count(void) { return launches(); }

int crava_gpu_create(const crava_gpu_params *params, int device, void *stream,
                     crava_gpu_ctx **out) {
  if (!out) return CRAVA_GPU_ERR_ARG;
  *out = nullptr;
  int rc = validate(params);
  if (rc) return rc;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) return CRAVA_GPU_ERR_NODEV;
  if (device < 0 || device >= ndev) return CRAVA_GPU_ERR_ARG;
  DeviceGuard guard(device);
  auto *c = new (std::nothrow) crava_gpu_ctx();
  if (!c) return CRAVA_GPU_ERR_ALLOC;
  c->device = device;
  c->stream = static_cast<cudaStream_t>(stream);
  c->p = *params;
  const int nt = params->ntheta, nzp = params->nzp;
  c->wavelet.assign(params->wavelet, params->wavelet + (size_t)nt * nzp);
  if (params->wavelet_norm) c->wnorm.assign(params->wavelet_norm, params->wavelet_norm + nt);
  c->A.assign(params->A, params->A + 3 * nt);
  c->theta.assign(params->theta_cov, params->theta_cov + nt * nt);
  c->var0.assign(params->var0, params->var0 + 9);
  c->p.wavelet = c->wavelet.data();
  c->p.wavelet_norm = c->wnorm.empty() ? nullptr : c->wnorm.data();
  c->p.A = c->A.data();
  c->p.theta_cov = c->theta.data();
  c->p.var0 = c->var0.data();
  c->g = Geom::make(params->nxp, params->nyp, params->nzp);
  c->consts.nt = nt;
  c->consts.wnc = params->wnc;
  c->consts.kappa_refine = kKappaRefineDefault;
  c->consts.solve_shape = -1;
  for (int l = 0; l < nt; ++l) {
    for (int q = 0; q < 3; ++q) c->consts.A[l][q] = c->A[3 * l + q];
    for (int m = 0; m < nt; ++m) c->consts.theta[l][m] = c->theta[l * nt + m];
  }
  const double *v = c->var0.data();
  c->consts.var0[0] = v[0]; c->consts.var0[1] = v[4]; c->consts.var0[2] = v[8];
  c->consts.var0[3] = v[1]; c->consts.var0[4] = v[2]; c->consts.var0[5] = v[5];

  auto fail = [&](int code) { crava_gpu_destroy(c); return code; };
  if ((rc = fft_plans_create(c->g, &c->plans))) return fail(rc);
  unit_plan(c->g, nt, &c->uplan);
  if ((rc = kz_tables_alloc(nzp, nt, &c->tables))) return fail(rc);
  if (cudaMalloc(&c->counters, sizeof(DevCounters)) != cudaSuccess) return fail(CRAVA_GPU_ERR_ALLOC);
  for (auto &e : c->ev)
    if (cudaEventCreate(&e) != cudaSuccess) return fail(CRAVA_GPU_ERR_CUDA);
  for (auto &ls : c->lane_s)
    if (cudaStreamCreateWithFlags(&ls, cudaStreamNonBlocking) != cudaSuccess) return fail(CRAVA_GPU_ERR_CUDA);
  if (cudaEventCreateWithFlags(&c->lane_fork, cudaEventDisableTiming) != cudaSuccess) return fail(CRAVA_GPU_ERR_CUDA);
  for (auto &e : c->lane_join)
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return fail(CRAVA_GPU_ERR_CUDA);
  if ((rc = kz_woodbury_alloc(nzp, (long long)c->g.cnxp * c->g.nyp, &c->tables))) return fail(rc);
  if ((rc = kz_tables_build(c->p, &c->tables, c->stream))) return fail(rc);
  if ((rc = kz_order_build(nzp, &c->tables, c->stream, &c->n_inverted))) return fail(rc);
  if ((rc = kz_woodbury_build(c->consts, nzp, c->tables, c->stream))) return fail(rc);
  // the flags of non-finite band-gated bins (ZPrior): one bit per bin and
  // the any-flag word, allocated here so that the unit allocates nothing
  // (and can be captured into a CUDA graph on its first call)
  if (z_prior_supported(c->plans)) {
    const long long words = (c->g.csize + 31) / 32;
    if (cudaMalloc(&c->gated_nf, (size_t)(words + 1) * sizeof(unsigned)) != cudaSuccess) {
      c->gated_nf = nullptr;
      return fail(CRAVA_GPU_ERR_ALLOC);
    }
    if (cudaMemset(c->gated_nf, 0, (size_t)(words + 1) * sizeof(unsigned)) != cudaSuccess) return fail(CRAVA_GPU_ERR_CUDA);
    c->gated_nf_words = words;
  }
  *out = c;
  return CRAVA_GPU_OK;
}

int crava_gpu_destroy(crava_gpu_ctx *c) {
  if (!c) return CRAVA_GPU_OK;
  DeviceGuard guard(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  else cudaDeviceSynchronize();
  if (c->s_out) cudaStreamSynchronize(c->s_out);
  if (c->s_in) cudaStreamSynchronize(c->s_in);
  for (auto &ls : c->lane_s) if (ls) cudaStreamSynchronize(ls);
  fft_plans_destroy(&c->plans);
  kz_tables_free(&c->tables);
  cudaFree(c->counters);
  cudaFree(c->work);
  cudaFree(c->W);
  cudaFree(c->synt_H);
  cudaFree(c->prior_buf);
  cudaFree(c->div_buf);
  cudaFree(c->ll_buf);
  cudaFree(c->gated_nf);
  if (c->ll_host) cudaFreeHost(c->ll_host);
  cudaFree(c->file_dev);
  if (c->file_host) cudaFreeHost(c->file_host);
  for (auto &e : c->ev) if (e) cudaEventDestroy(e);
  for (auto &e : c->grid_ev) if (e) cudaEventDestroy(e);
  for (auto &e : c->slot_done) if (e) cudaEventDestroy(e);
  for (auto &e : c->lane_join) if (e) cudaEventDestroy(e);
  if (c->lane_fork) cudaEventDestroy(c->lane_fork);
  for (auto &ls : c->lane_s) if (ls) cudaStreamDestroy(ls);
  for (auto &r : c->recs) { cudaEventDestroy(r.a); cudaEventDestroy(r.b); }
  for (auto &e : c->pool) cudaEventDestroy(e);
  if (c->s_in) cudaStreamDestroy(c->s_in);
  if (c->s_out) cudaStreamDestroy(c->s_out);
  delete c;
  return CRAVA_GPU_OK;
}

int crava_gpu_fft_r2c(crava_gpu_ctx *c, float *grid, int type) {
  if (check_ctx(c) || !grid || (reinterpret_cast<uintptr_t>(grid) & 7u)) return CRAVA_GPU_ERR_ARG;
  if (type < CRAVA_GRID_DATA || type > CRAVA_GRID_COVARIANCE) return CRAVA_GPU_ERR_ARG;
  DeviceGuard guard(c->device);
  return pass_forward(c, grid, grid, type);
}

int crava_gpu_fft_c2r(crava_gpu_ctx *c, float *grid, int type) {
  if (check_ctx(c) || !grid || (reinterpret_cast<uintptr_t>(grid) & 7u)) return CRAVA_GPU_ERR_ARG;
  if (type < CRAVA_GRID_DATA || type > CRAVA_GRID_COVARIANCE) return CRAVA_GPU_ERR_ARG;
  DeviceGuard guard(c->device);
  return pass_inverse(c, grid, type);
}

int crava_gpu_fft_xy(crava_gpu_ctx *c, float *grid, int dir, int type, int nzp_full) {
  if (check_ctx(c) || !grid || (reinterpret_cast<uintptr_t>(grid) & 7u)) return CRAVA_GPU_ERR_ARG;
  if ((dir != -1 && dir != 1) || type < CRAVA_GRID_DATA || type > CRAVA_GRID_COVARIANCE) return CRAVA_GPU_ERR_ARG;
  if (nzp_full < c->g.nzp) return CRAVA_GPU_ERR_ARG;
  DeviceGuard guard(c->device);
  // the scale of the whole grid, rounded exactly as the 3-D transforms round it
  const Geom full = Geom::make(c->g.nxp, c->g.nyp, nzp_full);
  const float scale = dir < 0 ? forward_scale(full, type) : inverse_scale(full, type);
  int rc;
  // the same x and y kernels as the 3-D transforms of this geometry
  if (use_plane_xy(c->plans)) return plane_xy(c->plans, grid, grid, dir, scale, nullptr, c->stream);
  if (dir < 0) {
    if ((rc = fft_rows(c->plans, grid, -1, scale, c->stream))) return rc;
    return fft_cols_y(c->plans, reinterpret_cast<float2 *>(grid), -1, c->stream);
  }
  if ((rc = fft_cols_y(c->plans, reinterpret_cast<float2 *>(grid), 1, c->stream))) return rc;
  return fft_rows(c->plans, grid, 1, scale, c->stream);
}

int crava_gpu_fft_z(crava_gpu_ctx *c, float *grid, int dir) {
  if (check_ctx(c) || !grid || (reinterpret_cast<uintptr_t>(grid) & 7u)) return CRAVA_GPU_ERR_ARG;
  if (dir != -1 && dir != 1) return CRAVA_GPU_ERR_ARG;
  DeviceGuard guard(c->device);
  return fft_cols_z(c->plans, reinterpret_cast<float2 *>(grid), dir, c->stream);
}

int crava_gpu_posterior(crava_gpu_ctx *c, const crava_gpu_grids *gr, int precision) {
  int rc;
  if ((rc = check_ctx(c)) || (rc = check_grids(c, gr))) return rc;
  if (!valid_precision(precision)) return CRAVA_GPU_ERR_ARG;
  DeviceGuard guard(c->device);
  CRAVA_CUDA_TRY(cudaMemsetAsync(c->counters, 0, sizeof(DevCounters), c->stream));
  CRAVA_CUDA_TRY(cudaEventRecord(c->ev[0], c->stream));
  CRAVA_CUDA_TRY(cudaEventRecord(c->ev[1], c->stream));
  if ((rc = pass_solve(c, gr, precision))) return rc;
  CRAVA_CUDA_TRY(cudaEventRecord(c->ev[2], c->stream));
  CRAVA_CUDA_TRY(cudaEventRecord(c->ev[3], c->stream));
  c->timed = true;
  return CRAVA_GPU_OK;
}

int crava_gpu_posterior_unit(crava_gpu_ctx *c, const crava_gpu_grids *gr, int precision) {
  int rc;
  if ((rc = check_ctx(c)) || (rc = check_grids(c, gr))) return rc;
  if (!valid_precision(precision)) return CRAVA_GPU_ERR_ARG;
  DeviceGuard guard(c->device);
  return run_unit(c, gr, gr, precision);
}

int crava_gpu_posterior_unit_oop(crava_gpu_ctx *c, const crava_gpu_grids *in,
                                 const crava_gpu_grids *out, int precision) {
  int rc;
  if ((rc = check_ctx(c)) || (rc = check_grids(c, in)) || (rc = check_grids(c, out))) return rc;
  if (!valid_precision(precision)) return CRAVA_GPU_ERR_ARG;
  DeviceGuard guard(c->device);
  return run_unit(c, in, out, precision);
}

int crava_gpu_set_fused(crava_gpu_ctx *c, int enable) {
  if (check_ctx(c)) return CRAVA_GPU_ERR_ARG;
  c->fused = enable != 0;
  return CRAVA_GPU_OK;
}

int crava_gpu_fused_available(crava_gpu_ctx *c, int precision) {
  if (check_ctx(c)) return 0;
  return c->uplan.ok && precision != CRAVA_SOLVE_FP32;
}

int crava_gpu_set_profiling(crava_gpu_ctx *c, int enable) {
  if (check_ctx(c)) return CRAVA_GPU_ERR_ARG;
  c->prof = enable != 0;
  return CRAVA_GPU_OK;
}

int crava_gpu_get_profile(crava_gpu_ctx *c, crava_gpu_kernel_profile *out, int max, int *count) {
  if (check_ctx(c) || !count || (max > 0 && !out)) return CRAVA_GPU_ERR_ARG;
  DeviceGuard guard(c->device);
  CRAVA_CUDA_TRY(cudaStreamSynchronize(c->stream));
  prof_collect(c);
  int n = 0;
  for (int k = 0; k < K_NKINDS; ++k) {
    if (!c->prof_n[k]) continue;
    if (n < max) {
      crava_gpu_kernel_profile &o = out[n];
      std::memset(&o, 0, sizeof o);
      std::snprintf(o.name, sizeof o.name, "%s", kKindName[k]);
      o.launches = c->prof_n[k];
      o.total_ms = c->prof_ms[k];
      o.bytes_per_launch = c->prof_bytes[k] / (double)c->prof_n[k];
    }
    ++n;
  }
  *count = n;
  for (int k = 0; k < K_NKINDS; ++k) { c->prof_ms[k] = 0.0; c->prof_bytes[k] = 0.0; c->prof_n[k] = 0; }
  return CRAVA_GPU_OK;
}

int crava_gpu_host_register(void *ptr, uint64_t bytes) {
  if (!ptr || !bytes) return CRAVA_GPU_ERR_ARG;
  cudaError_t e = cudaHostRegister(ptr, (size_t)bytes, cudaHostRegisterDefault);
  if (e != cudaSuccess) { set_last_error(e, "cudaHostRegister", __FILE__, __LINE__); return CRAVA_GPU_ERR_CUDA; }
  return CRAVA_GPU_OK;
}

int crava_gpu_host_unregister(void *ptr) {
  if (!ptr) return CRAVA_GPU_ERR_ARG;
  cudaError_t e = cudaHostUnregister(ptr);
  if (e != cudaSuccess) { set_last_error(e, "cudaHostUnregister", __FILE__, __LINE__); return CRAVA_GPU_ERR_CUDA; }
  return CRAVA_GPU_OK;
}

}  // extern "C"

namespace crava {

// Device work grids for the host-buffer path: `slots` sets of (10 + nt)
// grids, copy streams and events (reallocated when more slots are needed).
static int ensure_host_work(crava_gpu_ctx *c, int slots) {
  const int ngrid = 10 + c->p.ntheta;
  const size_t gbytes = (size_t)c->g.rsize * sizeof(float);
  if (c->work_slots < slots) {
    if (c->work) {
      CRAVA_CUDA_TRY(cudaDeviceSynchronize());
      cudaFree(c->work);
      c->work = nullptr;
      c->work_slots = 0;
    }
    if (cudaMalloc(&c->work, gbytes * ngrid * slots) != cudaSuccess) { c->work = nullptr; return CRAVA_GPU_ERR_ALLOC; }
    c->work_slots = slots;
  }
  if (!c->s_in) {
    CRAVA_CUDA_TRY(cudaStreamCreateWithFlags(&c->s_in, cudaStreamNonBlocking));
    CRAVA_CUDA_TRY(cudaStreamCreateWithFlags(&c->s_out, cudaStreamNonBlocking));
    c->grid_ev.assign(2 * ngrid + 1, nullptr);
    for (auto &e : c->grid_ev) CRAVA_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    for (auto &e : c->slot_done) CRAVA_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  }
  return CRAVA_GPU_OK;
}

// One host-buffer unit on work slot `slot`: uploads `in` (each grid's
// copy overlapping the transforms of those before it), solves, and
// downloads the outputs into `out` (each grid as soon as its inverse
// transform is done).  Stream-ordered, returns once enqueued.
static int enqueue_unit_host(crava_gpu_ctx *c, const crava_gpu_grids *hin, const crava_gpu_grids *hout,
                             int precision, int slot, bool order_after_compute) {
  int rc;
  const int nt = c->p.ntheta, ngrid = 10 + nt;
  const size_t gbytes = (size_t)c->g.rsize * sizeof(float);
  crava_gpu_grids dg{};
  std::vector<const float *> hsrc(ngrid);
  std::vector<float *> hdst(ngrid), dev(ngrid);
  std::vector<int> type(ngrid);
  int i = 0;
  for (int q = 0; q < 3; ++q, ++i) { hsrc[i] = hin->mu[q]; hdst[i] = hout->mu[q]; type[i] = CRAVA_GRID_PARAMETER; }
  for (int l = 0; l < nt; ++l, ++i) { hsrc[i] = hin->data[l]; hdst[i] = hout->data[l]; type[i] = CRAVA_GRID_DATA; }
  for (int t = 0; t < 6; ++t, ++i) { hsrc[i] = hin->cov[t]; hdst[i] = hout->cov[t]; type[i] = CRAVA_GRID_COVARIANCE; }
  hsrc[i] = hin->err_corr; hdst[i] = hout->err_corr; type[i] = CRAVA_GRID_COVARIANCE;
  float *base = c->work + (size_t)slot * ngrid * c->g.rsize;
  for (int k = 0; k < ngrid; ++k) dev[k] = base + (size_t)k * c->g.rsize;
  i = 0;
  for (int q = 0; q < 3; ++q) dg.mu[q] = dev[i++];
  for (int l = 0; l < nt; ++l) dg.data[l] = dev[i++];
  for (int t = 0; t < 6; ++t) dg.cov[t] = dev[i++];
  dg.err_corr = dev[i];

  const cudaStream_t s = c->stream;
  CRAVA_CUDA_TRY(cudaMemsetAsync(c->counters, 0, sizeof(DevCounters), s));
  CRAVA_CUDA_TRY(cudaEventRecord(c->ev[0], s));
  if (order_after_compute) {
    // the copy stream must not overtake earlier work on the compute stream
    CRAVA_CUDA_TRY(cudaEventRecord(c->grid_ev[2 * ngrid], s));
    CRAVA_CUDA_TRY(cudaStreamWaitEvent(c->s_in, c->grid_ev[2 * ngrid], 0));
  }
  // the slot's grids are free once the step that used them last has
  // downloaded its outputs
  CRAVA_CUDA_TRY(cudaStreamWaitEvent(c->s_in, c->slot_done[slot], 0));
  const bool fused = use_fused(c, precision);
  if (fused && (rc = ensure_workspace(c))) return rc;
  ZPrior zp[6];
  bool gated = false;  // the band-gated covariance rule in the forward z passes
  if (!fused && (rc = gated_prior_setup(c, precision, zp, &gated))) return rc;
  const double gb = (double)c->g.csize * 8.0, wb = (double)c->uplan.wgrid * 8.0;
  for (int k = 0; k < ngrid; ++k) {
    CRAVA_CUDA_TRY(cudaMemcpyAsync(dev[k], hsrc[k], gbytes, cudaMemcpyHostToDevice, c->s_in));
    CRAVA_CUDA_TRY(cudaEventRecord(c->grid_ev[k], c->s_in));
    CRAVA_CUDA_TRY(cudaStreamWaitEvent(s, c->grid_ev[k], 0));
    if (fused) {
      Scope sc(c, K_PLANE_FWD, gb + wb);
      float2 *wk = c->W + (size_t)k * c->uplan.wgrid;
      const float fsc = forward_scale(c->g, type[k]);
      const float *src = dev[k];
      if ((rc = unit_plane_forward(c->uplan, c->plans, &src, &wk, &fsc, 1, s))) return rc;
    } else if ((rc = pass_forward(c, dev[k], dev[k], type[k],
                                  gated && k >= 3 + nt && k < 9 + nt ? &zp[k - 3 - nt] : nullptr))) {
      return rc;
    }
  }
  if (gated && (rc = gated_prior_count(c))) return rc;
  CRAVA_CUDA_TRY(cudaEventRecord(c->ev[1], s));
  if (fused) {
    float2 *w[kMaxUnitGrids];
    for (int k = 0; k < ngrid; ++k) w[k] = c->W + (size_t)k * c->uplan.wgrid;
    Scope sc(c, K_ZSOLVE, (2 * ngrid - 1) * wb);
    if ((rc = unit_zsolve(c->uplan, c->plans, c->consts, c->tables, w, precision, c->counters, s))) return rc;
  } else if ((rc = pass_solve(c, &dg, precision, gated))) {
    return rc;
  }
  CRAVA_CUDA_TRY(cudaEventRecord(c->ev[2], s));
  for (int k = 0; k < ngrid - 1; ++k) {  // the noise correlation is not an output
    if (fused) {
      Scope sc(c, K_PLANE_INV, gb + wb);
      const float2 *wk = c->W + (size_t)k * c->uplan.wgrid;
      const float isc = inverse_scale(c->g, type[k]);
      if ((rc = unit_plane_inverse(c->uplan, c->plans, &wk, &dev[k], &isc, nullptr, 1, s))) return rc;
    } else if ((rc = pass_inverse(c, dev[k], type[k]))) {
      return rc;
    }
    CRAVA_CUDA_TRY(cudaEventRecord(c->grid_ev[ngrid + k], s));
    CRAVA_CUDA_TRY(cudaStreamWaitEvent(c->s_out, c->grid_ev[ngrid + k], 0));
    CRAVA_CUDA_TRY(cudaMemcpyAsync(hdst[k], dev[k], gbytes, cudaMemcpyDeviceToHost, c->s_out));
  }
  CRAVA_CUDA_TRY(cudaEventRecord(c->ev[3], s));
  CRAVA_CUDA_TRY(cudaEventRecord(c->slot_done[slot], c->s_out));
  c->timed = true;
  return CRAVA_GPU_OK;
}

}  // namespace crava

extern "C" {

int crava_gpu_posterior_unit_host(crava_gpu_ctx *c, const crava_gpu_grids *hg, int precision) {
  int rc;
  if ((rc = check_ctx(c)) || (rc = check_grids(c, hg))) return rc;
  if (!valid_precision(precision)) return CRAVA_GPU_ERR_ARG;
  DeviceGuard guard(c->device);
  if ((rc = ensure_host_work(c, 1))) return rc;
  if ((rc = enqueue_unit_host(c, hg, hg, precision, 0, true))) return rc;
  CRAVA_CUDA_TRY(cudaStreamSynchronize(c->s_out));
  CRAVA_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return CRAVA_GPU_OK;
}

int crava_gpu_posterior_unit_host_async(crava_gpu_ctx *c, const crava_gpu_grids *hin,
                                        const crava_gpu_grids *hout, int precision) {
  int rc;
  if ((rc = check_ctx(c)) || (rc = check_grids(c, hin)) || (rc = check_grids(c, hout))) return rc;
  if (!valid_precision(precision)) return CRAVA_GPU_ERR_ARG;
  DeviceGuard guard(c->device);
  if ((rc = ensure_host_work(c, 2))) return rc;
  const int slot = (int)(c->host_seq & 1);
  if ((rc = enqueue_unit_host(c, hin, hout, precision, slot, c->host_seq == 0))) return rc;
  ++c->host_seq;
  return CRAVA_GPU_OK;
}

int crava_gpu_host_wait(crava_gpu_ctx *c) {
  if (check_ctx(c)) return CRAVA_GPU_ERR_ARG;
  DeviceGuard guard(c->device);
  if (c->s_out) CRAVA_CUDA_TRY(cudaStreamSynchronize(c->s_out));
  if (c->s_in) CRAVA_CUDA_TRY(cudaStreamSynchronize(c->s_in));
  CRAVA_CUDA_TRY(cudaStreamSynchronize(c->stream));
  c->host_seq = 0;
  return CRAVA_GPU_OK;
}

int crava_gpu_noise_fill(crava_gpu_ctx *c, float *grid, uint64_t seed, uint64_t stream_id) {
  if (check_ctx(c) || !grid || (reinterpret_cast<uintptr_t>(grid) & 7u)) return CRAVA_GPU_ERR_ARG;
  DeviceGuard guard(c->device);
  return noise_fill(c->g, reinterpret_cast<float2 *>(grid), seed, stream_id, c->stream);
}

int crava_gpu_sim_filter(crava_gpu_ctx *c, const float *const cov[6], float *const seed[3]) {
  if (check_ctx(c) || !cov || !seed) return CRAVA_GPU_ERR_ARG;
  const float2 *cv[6];
  float2 *sd[3];
  for (int t = 0; t < 6; ++t) {
    if (!cov[t] || (reinterpret_cast<uintptr_t>(cov[t]) & 7u)) return CRAVA_GPU_ERR_ARG;
    cv[t] = reinterpret_cast<const float2 *>(cov[t]);
  }
  for (int q = 0; q < 3; ++q) {
    if (!seed[q] || (reinterpret_cast<uintptr_t>(seed[q]) & 7u)) return CRAVA_GPU_ERR_ARG;
    sd[q] = reinterpret_cast<float2 *>(seed[q]);
  }
  DeviceGuard guard(c->device);
  CRAVA_CUDA_TRY(cudaMemsetAsync(c->counters, 0, sizeof(DevCounters), c->stream));
  c->timed = false;
  return sim_filter(c->g, cv, sd, c->counters, c->stream);
}

int crava_gpu_simulate(crava_gpu_ctx *c, const float *const cov[6], const float *const post_mean[3],
                       uint64_t seed, int first_index, int count, float *const *out) {
  if (check_ctx(c) || !cov || !post_mean || !out || count < 0 || first_index < 0) return CRAVA_GPU_ERR_ARG;
  const float2 *cv[6];
  for (int t = 0; t < 6; ++t) {
    if (!cov[t] || (reinterpret_cast<uintptr_t>(cov[t]) & 7u)) return CRAVA_GPU_ERR_ARG;
    cv[t] = reinterpret_cast<const float2 *>(cov[t]);
  }
  for (int q = 0; q < 3; ++q)
    if (!post_mean[q] || (reinterpret_cast<uintptr_t>(post_mean[q]) & 7u)) return CRAVA_GPU_ERR_ARG;
  for (int r = 0; r < 3 * count; ++r)
    if (!out[r] || (reinterpret_cast<uintptr_t>(out[r]) & 7u)) return CRAVA_GPU_ERR_ARG;
  DeviceGuard guard(c->device);
  const cudaStream_t s = c->stream;
  int rc;
  CRAVA_CUDA_TRY(cudaMemsetAsync(c->counters, 0, sizeof(DevCounters), s));
  CRAVA_CUDA_TRY(cudaEventRecord(c->ev[0], s));
  if ((rc = simulate_batches(c, cv, post_mean, seed, (uint64_t)first_index, count, out, nullptr, 0)))
    return rc;
  CRAVA_CUDA_TRY(cudaEventRecord(c->ev[1], s));
  CRAVA_CUDA_TRY(cudaEventRecord(c->ev[2], s));
  CRAVA_CUDA_TRY(cudaEventRecord(c->ev[3], s));
  c->timed = true;
  return CRAVA_GPU_OK;
}

int crava_gpu_get_stats(crava_gpu_ctx *c, crava_gpu_stats *st) {
  if (check_ctx(c) || !st) return CRAVA_GPU_ERR_ARG;
  DeviceGuard guard(c->device);
  CRAVA_CUDA_TRY(cudaStreamSynchronize(c->stream));
  DevCounters h{};
  CRAVA_CUDA_TRY(cudaMemcpy(&h, c->counters, sizeof h, cudaMemcpyDeviceToHost));
  std::memset(st, 0, sizeof *st);
  st->chol_fail_bins = (long long)h.chol_fail;
  st->nonfinite_bins = (long long)h.nonfinite;
  st->refined_bins = (long long)h.refined;
  unsigned long long waits = 0;
  if (tile_wait_timeouts(&waits)) return CRAVA_GPU_ERR_CUDA;
  st->tile_wait_timeouts = (long long)waits;
  if (c->timed) {
    cudaEventElapsedTime(&st->ms_forward, c->ev[0], c->ev[1]);
    cudaEventElapsedTime(&st->ms_solve, c->ev[1], c->ev[2]);
    cudaEventElapsedTime(&st->ms_inverse, c->ev[2], c->ev[3]);
    cudaEventElapsedTime(&st->ms_total, c->ev[0], c->ev[3]);
  }
  return CRAVA_GPU_OK;
}

int crava_gpu_kz_tables(crava_gpu_ctx *c, float *wd, float *e1, float *e2, float *e3, int *inv) {
  if (check_ctx(c) || !wd || !e1 || !e2 || !e3 || !inv) return CRAVA_GPU_ERR_ARG;
  DeviceGuard guard(c->device);
  const size_t n = (size_t)c->p.nzp * c->p.ntheta;
  CRAVA_CUDA_TRY(cudaStreamSynchronize(c->stream));
  CRAVA_CUDA_TRY(cudaMemcpy(wd, c->tables.wd, n * sizeof(float2), cudaMemcpyDeviceToHost));
  CRAVA_CUDA_TRY(cudaMemcpy(e1, c->tables.e1, n * sizeof(float2), cudaMemcpyDeviceToHost));
  CRAVA_CUDA_TRY(cudaMemcpy(e2, c->tables.e2, n * sizeof(float2), cudaMemcpyDeviceToHost));
  CRAVA_CUDA_TRY(cudaMemcpy(e3, c->tables.e3, n * sizeof(float), cudaMemcpyDeviceToHost));
  CRAVA_CUDA_TRY(cudaMemcpy(inv, c->tables.inv, (size_t)c->p.nzp * sizeof(int), cudaMemcpyDeviceToHost));
  return CRAVA_GPU_OK;
}

int crava_gpu_set_kz_tables(crava_gpu_ctx *c, const float *wd, const float *e1, const float *e2,
                            const float *e3, const int *inv) {
  if (check_ctx(c) || !wd || !e1 || !e2 || !e3 || !inv) return CRAVA_GPU_ERR_ARG;
  DeviceGuard guard(c->device);
  const size_t n = (size_t)c->p.nzp * c->p.ntheta;
  CRAVA_CUDA_TRY(cudaStreamSynchronize(c->stream));
  CRAVA_CUDA_TRY(cudaMemcpy(c->tables.wd, wd, n * sizeof(float2), cudaMemcpyHostToDevice));
  CRAVA_CUDA_TRY(cudaMemcpy(c->tables.e1, e1, n * sizeof(float2), cudaMemcpyHostToDevice));
  CRAVA_CUDA_TRY(cudaMemcpy(c->tables.e2, e2, n * sizeof(float2), cudaMemcpyHostToDevice));
  CRAVA_CUDA_TRY(cudaMemcpy(c->tables.e3, e3, n * sizeof(float), cudaMemcpyHostToDevice));
  CRAVA_CUDA_TRY(cudaMemcpy(c->tables.inv, inv, (size_t)c->p.nzp * sizeof(int), cudaMemcpyHostToDevice));
  int rc = kz_order_build(c->p.nzp, &c->tables, c->stream, &c->n_inverted);
  if (rc) return rc;
  return kz_woodbury_build(c->consts, c->p.nzp, c->tables, c->stream);
}

}  // extern "C"
