// batch.cu -- launch-shape autotuner and the vintage batch: several
// posterior units with their realisations, captured once into a CUDA graph
// and replayed with one launch per run.
#include <vector>

#include "context.cuh"

using namespace crava;

struct crava_gpu_batch {
  struct Vintage {
    crava_gpu_ctx *ctx;
    crava_gpu_grids in, out;
    int precision;
    int nsim;
    uint64_t seed, first;
    std::vector<float *> sim;
    float2 **d_sim = nullptr;  // device copy of sim (the persistent filter's output table)
  };
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  bool graph_mode = true;
  std::vector<Vintage> v;
  std::vector<crava_gpu_ctx *> ctxs;    // distinct contexts
  std::vector<cudaStream_t> cstream;    // one branch stream per context
  cudaEvent_t fork = nullptr;
  std::vector<cudaEvent_t> join;
  unsigned long long *epoch = nullptr;  // device: runs completed
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  long long kernels = 0;                // kernel nodes per run
};

namespace {

__global__ void k_epoch_advance(unsigned long long *e) { *e += 1ull; }

bool aligned8(const void *p) { return p && (reinterpret_cast<uintptr_t>(p) & 7u) == 0; }

// Grid pointers of a crava_gpu_grids (mu, data, cov, err) in a flat list.
int grid_list(const crava_gpu_ctx *c, const crava_gpu_grids *g, const float **out) {
  int n = 0;
  for (int q = 0; q < 3; ++q) out[n++] = g->mu[q];
  for (int l = 0; l < c->p.ntheta; ++l) out[n++] = g->data[l];
  for (int t = 0; t < 6; ++t) out[n++] = g->cov[t];
  out[n++] = g->err_corr;
  return n;
}

// true when no grid of `in` is also a grid of `out` (byte ranges disjoint).
bool disjoint(const crava_gpu_ctx *c, const crava_gpu_grids *in, const crava_gpu_grids *out) {
  const float *a[kMaxUnitGrids], *b[kMaxUnitGrids];
  const int n = grid_list(c, in, a);
  grid_list(c, out, b);
  const uintptr_t bytes = (uintptr_t)c->g.rsize * sizeof(float);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      const uintptr_t x = reinterpret_cast<uintptr_t>(a[i]), y = reinterpret_cast<uintptr_t>(b[j]);
      if (x < y + bytes && y < x + bytes) return false;
    }
  return true;
}

// One vintage on its context's stream, up to its realisations.  Without
// realisations this is the whole unit (fused or three-pass, as tuned); with
// them it follows the reference's order: the covariance spectra stay in
// the Fourier domain until the realisations are drawn
// (src/crava.cpp:1165-1181, 1415-1599), so this part ends after the
// inverse transforms of the means and residuals.
int run_vintage_head(const crava_gpu_batch::Vintage &v) {
  crava_gpu_ctx *c = v.ctx;
  if (v.nsim == 0) return run_unit(c, &v.in, &v.out, v.precision);
  const int nt = c->p.ntheta;
  const crava_gpu_grids &in = v.in, &out = v.out;
  int rc;
  CRAVA_CUDA_TRY(cudaMemsetAsync(c->counters, 0, sizeof(DevCounters), c->stream));
  if ((rc = stage_event(c, 0))) return rc;
  for (int q = 0; q < 3; ++q)
    if ((rc = pass_forward(c, in.mu[q], out.mu[q], CRAVA_GRID_PARAMETER))) return rc;
  for (int l = 0; l < nt; ++l)
    if ((rc = pass_forward(c, in.data[l], out.data[l], CRAVA_GRID_DATA))) return rc;
  // the band-gated covariance rule in the forward z passes (as run_unit)
  ZPrior zp[6];
  bool gated = false;
  if ((rc = gated_prior_setup(c, v.precision, zp, &gated))) return rc;
  for (int t = 0; t < 6; ++t)
    if ((rc = pass_forward(c, in.cov[t], out.cov[t], CRAVA_GRID_COVARIANCE, gated ? &zp[t] : nullptr))) return rc;
  if ((rc = pass_forward(c, in.err_corr, out.err_corr, CRAVA_GRID_COVARIANCE))) return rc;
  if (gated && (rc = gated_prior_count(c))) return rc;
  if ((rc = stage_event(c, 1))) return rc;
  if ((rc = pass_solve(c, &out, v.precision, gated))) return rc;
  if ((rc = stage_event(c, 2))) return rc;
  for (int q = 0; q < 3; ++q)
    if ((rc = pass_inverse(c, out.mu[q], CRAVA_GRID_PARAMETER))) return rc;
  for (int l = 0; l < nt; ++l)
    if ((rc = pass_inverse(c, out.data[l], CRAVA_GRID_DATA))) return rc;
  return CRAVA_GPU_OK;
}

// The rest of a vintage with realisations, after the batch's realisation
// filter: each realisation's three inverse transforms with the posterior
// mean added, then the inverse transforms of the covariances.
int run_vintage_tail(const crava_gpu_batch::Vintage &v) {
  crava_gpu_ctx *c = v.ctx;
  if (v.nsim == 0) return CRAVA_GPU_OK;
  const crava_gpu_grids &out = v.out;
  int rc;
  const float *pm[3] = {out.mu[0], out.mu[1], out.mu[2]};
  if ((rc = inverse_realisations(c, v.sim.data(), 3 * v.nsim, pm))) return rc;
  for (int t = 0; t < 6; ++t)
    if ((rc = pass_inverse(c, out.cov[t], CRAVA_GRID_COVARIANCE))) return rc;
  if ((rc = stage_event(c, 3))) return rc;
  c->timed = !c->capture;
  return CRAVA_GPU_OK;
}

// The realisation filter of every vintage with realisations, one
// persistent launch on the batch stream (noise_filter_vintages).
int filter_vintages(crava_gpu_batch *b) {
  SimVintage sv[kMaxSimVintages];
  int nv = 0;
  for (const auto &v : b->v) {
    if (v.nsim == 0) continue;
    if (nv == kMaxSimVintages) return CRAVA_GPU_ERR_ARG;
    crava_gpu_ctx *c = v.ctx;
    SimVintage &w = sv[nv++];
    for (int t = 0; t < 6; ++t) w.cov[t] = reinterpret_cast<const float2 *>(v.out.cov[t]);
    w.out = v.d_sim;
    w.csize = c->g.csize;
    w.cnxp = c->g.cnxp; w.nyp = c->g.nyp; w.nzp = c->g.nzp;
    w.nsim = v.nsim;
    w.seed = v.seed;
    w.stream0 = 3ull * v.first;
    w.epoch_mul = 3ull * (unsigned long long)v.nsim;
    w.counters = c->counters;
  }
  if (nv == 0) return CRAVA_GPU_OK;
  int rc = noise_filter_vintages(sv, nv, b->epoch, b->stream);
  if (!rc) note_launch();
  return rc;
}

// Enqueues one run: fork from the batch stream into one branch per
// context, the vintages, join, and (advance) the epoch counter.
int enqueue(crava_gpu_batch *b, bool capture, bool advance) {
  const size_t nc = b->ctxs.size();
  std::vector<cudaStream_t> saved(nc);
  for (size_t i = 0; i < nc; ++i) {
    saved[i] = b->ctxs[i]->stream;
    b->ctxs[i]->stream = b->cstream[i];
    b->ctxs[i]->capture = capture;
  }
  int rc = CRAVA_GPU_OK;
  cudaError_t e = cudaEventRecord(b->fork, b->stream);
  for (size_t i = 0; i < nc && e == cudaSuccess; ++i) e = cudaStreamWaitEvent(b->cstream[i], b->fork, 0);
  if (e != cudaSuccess) {
    set_last_error(e, "batch fork", __FILE__, __LINE__);
    rc = CRAVA_GPU_ERR_CUDA;
  }
  auto join = [&]() {
    for (size_t i = 0; i < nc && !rc; ++i) {
      e = cudaEventRecord(b->join[i], b->cstream[i]);
      if (e == cudaSuccess) e = cudaStreamWaitEvent(b->stream, b->join[i], 0);
      if (e != cudaSuccess) {
        set_last_error(e, "batch join", __FILE__, __LINE__);
        rc = CRAVA_GPU_ERR_CUDA;
      }
    }
  };
  // the vintages up to their realisations, one branch per context
  for (size_t k = 0; k < b->v.size() && !rc; ++k) rc = run_vintage_head(b->v[k]);
  bool sims = false;
  for (const auto &v : b->v) sims = sims || v.nsim > 0;
  if (sims && !rc) {
    // every vintage's realisation filter in one persistent launch on the
    // batch stream, then the branches again for the realisations' inverse
    // transforms and the covariances
    join();
    if (!rc) rc = filter_vintages(b);
    if (!rc) {
      e = cudaEventRecord(b->fork, b->stream);
      for (size_t i = 0; i < nc && e == cudaSuccess; ++i) e = cudaStreamWaitEvent(b->cstream[i], b->fork, 0);
      if (e != cudaSuccess) {
        set_last_error(e, "batch fork", __FILE__, __LINE__);
        rc = CRAVA_GPU_ERR_CUDA;
      }
    }
    for (size_t k = 0; k < b->v.size() && !rc; ++k) rc = run_vintage_tail(b->v[k]);
  }
  join();
  if (!rc && advance) {
    k_epoch_advance<<<1, 1, 0, b->stream>>>(b->epoch);
    cudaError_t le = cudaGetLastError();
    if (le != cudaSuccess) {
      set_last_error(le, "kernel launch", __FILE__, __LINE__);
      rc = CRAVA_GPU_ERR_CUDA;
    } else {
      note_launch();
    }
  }
  for (size_t i = 0; i < nc; ++i) {
    b->ctxs[i]->stream = saved[i];
    b->ctxs[i]->capture = false;
  }
  return rc;
}

void batch_free(crava_gpu_batch *b) {
  if (!b) return;
  DeviceGuard guard(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  for (cudaStream_t s : b->cstream) if (s) { cudaStreamSynchronize(s); cudaStreamDestroy(s); }
  for (cudaEvent_t e : b->join) if (e) cudaEventDestroy(e);
  if (b->fork) cudaEventDestroy(b->fork);
  if (b->epoch) cudaFree(b->epoch);
  for (auto &v : b->v) if (v.d_sim) cudaFree(v.d_sim);
  if (b->own_stream && b->stream) cudaStreamDestroy(b->stream);
  delete b;
}

}  // namespace

extern "C" {

int crava_gpu_get_tuning(crava_gpu_ctx *c, crava_gpu_tuning *out) {
  if (!c || !out) return CRAVA_GPU_ERR_ARG;
  out->cols_y_tile = c->plans.tile_y;
  out->cols_z_tile = c->plans.tile_z;
  out->fused = c->fused ? 1 : 0;
  out->ms = 0.0f;
  out->lanes = c->lanes;
  out->rows_x = c->plans.rows_x;
  out->kappa_refine = c->consts.kappa_refine;
  out->xy_fused = c->plans.plane_xy;
  out->solve_shape = c->consts.solve_shape;
  return CRAVA_GPU_OK;
}

int crava_gpu_set_tuning(crava_gpu_ctx *c, const crava_gpu_tuning *t) {
  if (!c || !t) return CRAVA_GPU_ERR_ARG;
  auto ok = [](int x) { return x == -1 || x == 0 || x == 1 || x == 8 || x == 16; };
  if (!ok(t->cols_y_tile) || !(ok(t->cols_z_tile) || t->cols_z_tile == 2)) return CRAVA_GPU_ERR_ARG;
  if (t->rows_x < -1 || t->rows_x > 1) return CRAVA_GPU_ERR_ARG;
  if (!(t->kappa_refine >= 0.0f)) return CRAVA_GPU_ERR_ARG;
  if (t->xy_fused < -1 || t->xy_fused > 1) return CRAVA_GPU_ERR_ARG;
  if (t->solve_shape < -1 || t->solve_shape > 8) return CRAVA_GPU_ERR_ARG;
  if (t->lanes < 1 || t->lanes > crava_gpu_ctx::kMaxLanes) return CRAVA_GPU_ERR_ARG;
  c->plans.tile_y = t->cols_y_tile;
  c->plans.tile_z = t->cols_z_tile;
  c->fused = t->fused != 0;
  c->lanes = t->lanes;
  c->plans.rows_x = t->rows_x;
  c->consts.kappa_refine = t->kappa_refine;
  c->plans.plane_xy = t->xy_fused;
  c->consts.solve_shape = t->solve_shape;
  return CRAVA_GPU_OK;
}

int crava_gpu_autotune(crava_gpu_ctx *c, const crava_gpu_grids *in, const crava_gpu_grids *out,
                       int precision, int reps, crava_gpu_tuning *best) {
  int rc;
  if (!c || reps < 1 || reps > 100) return CRAVA_GPU_ERR_ARG;
  if ((rc = check_grids(c, in)) || (rc = check_grids(c, out))) return rc;
  if (!valid_precision(precision) || !disjoint(c, in, out)) return CRAVA_GPU_ERR_ARG;
  DeviceGuard guard(c->device);
  std::vector<crava_gpu_tuning> cand;
  const bool ty = cols_tunable(c->g.nyp), tz = cols_tunable(c->g.nzp);
  // column choices of a length: the register-resident pass where it
  // exists, the in-place pass with 16 and 8 columns, the ping-pong pass
  auto choices = [](int n, bool tunable) {
    std::vector<int> v;
    if (cols_rr(n)) v.push_back(1);
    if (tunable) { v.push_back(16); v.push_back(8); v.push_back(0); }
    if (v.empty()) v.push_back(-1);
    return v;
  };
  const std::vector<int> cy = choices(c->g.nyp, ty);
  std::vector<int> cz = choices(c->g.nzp, tz);
  // the TMA z pass, where the grids allow it
  bool tma = cols_z_tma_supported(c->g, in->err_corr) && cols_z_tma_supported(c->g, out->err_corr);
  for (int q = 0; q < 3; ++q) tma = tma && cols_z_tma_supported(c->g, in->mu[q]) && cols_z_tma_supported(c->g, out->mu[q]);
  for (int l = 0; l < c->p.ntheta; ++l)
    tma = tma && cols_z_tma_supported(c->g, in->data[l]) && cols_z_tma_supported(c->g, out->data[l]);
  for (int q = 0; q < 6; ++q) tma = tma && cols_z_tma_supported(c->g, in->cov[q]) && cols_z_tma_supported(c->g, out->cov[q]);
  if (tma) cz.insert(cz.begin(), 2);
  const bool xy = plane_xy_supported(c->g);
  for (int lanes = 1; lanes <= 3; ++lanes) {
    for (int a : cy)
      for (int z : cz) cand.push_back({a, z, 0, 0.0f, lanes, -1, c->consts.kappa_refine, 0, c->consts.solve_shape});
    // the fused x + y pass replaces the y pass: only the z choices matter
    if (xy)
      for (int z : cz) cand.push_back({-1, z, 0, 0.0f, lanes, -1, c->consts.kappa_refine, 1, c->consts.solve_shape});
  }
  // the fused unit does not use the column passes: one candidate
  if (c->uplan.ok && precision != CRAVA_SOLVE_FP32) cand.push_back({-1, -1, 1, 0.0f, 1, -1, c->consts.kappa_refine, 0, c->consts.solve_shape});
  crava_gpu_tuning saved;
  crava_gpu_get_tuning(c, &saved);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  CRAVA_CUDA_TRY(cudaEventCreate(&e0));
  if (cudaEventCreate(&e1) != cudaSuccess) { cudaEventDestroy(e0); return CRAVA_GPU_ERR_CUDA; }
  int ibest = -1;
  rc = CRAVA_GPU_OK;
  for (size_t i = 0; i < cand.size() && !rc; ++i) {
    crava_gpu_set_tuning(c, &cand[i]);
    if ((rc = run_unit(c, in, out, precision))) break;  // warm-up
    cudaError_t e = cudaEventRecord(e0, c->stream);
    for (int r = 0; r < reps && !rc && e == cudaSuccess; ++r) rc = run_unit(c, in, out, precision);
    if (!rc && e == cudaSuccess) e = cudaEventRecord(e1, c->stream);
    if (!rc && e == cudaSuccess) e = cudaEventSynchronize(e1);
    float ms = 0.0f;
    if (!rc && e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    if (!rc && e != cudaSuccess) { set_last_error(e, "autotune timing", __FILE__, __LINE__); rc = CRAVA_GPU_ERR_CUDA; }
    if (rc) break;
    cand[i].ms = ms / (float)reps;
    if (ibest < 0 || cand[i].ms < cand[ibest].ms) ibest = (int)i;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc || ibest < 0) {
    crava_gpu_set_tuning(c, &saved);
    return rc ? rc : CRAVA_GPU_ERR_STATE;
  }
  crava_gpu_set_tuning(c, &cand[ibest]);
  if (best) *best = cand[ibest];
  return CRAVA_GPU_OK;
}

int crava_gpu_batch_create(const crava_gpu_vintage *vin, int n, int flags, void *stream,
                           crava_gpu_batch **out) {
  if (!out) return CRAVA_GPU_ERR_ARG;
  *out = nullptr;
  if (!vin || n < 1 || (flags & ~(CRAVA_BATCH_AUTOTUNE | CRAVA_BATCH_NO_GRAPH))) return CRAVA_GPU_ERR_ARG;
  int with_sims = 0;
  for (int k = 0; k < n; ++k) with_sims += vin[k].nsim > 0;
  if (with_sims > kMaxSimVintages) return CRAVA_GPU_ERR_ARG;  // one persistent filter launch holds them
  int rc;
  const int dev = vin[0].ctx ? vin[0].ctx->device : -1;
  for (int k = 0; k < n; ++k) {
    const crava_gpu_vintage &v = vin[k];
    crava_gpu_ctx *c = v.ctx;
    if (!c || c->device != dev || c->prof) return CRAVA_GPU_ERR_ARG;
    if ((rc = check_grids(c, &v.in)) || (rc = check_grids(c, &v.out))) return rc;
    if (!valid_precision(v.precision) || v.nsim < 0) return CRAVA_GPU_ERR_ARG;
    if (v.nsim > 0 && !v.sim_out) return CRAVA_GPU_ERR_ARG;
    for (int r = 0; r < 3 * v.nsim; ++r)
      if (!aligned8(v.sim_out[r])) return CRAVA_GPU_ERR_ARG;
    // in place would transform the inputs again on every run
    if (!disjoint(c, &v.in, &v.out)) return CRAVA_GPU_ERR_ARG;
  }
  DeviceGuard guard(dev);
  auto *b = new (std::nothrow) crava_gpu_batch();
  if (!b) return CRAVA_GPU_ERR_ALLOC;
  b->device = dev;
  b->graph_mode = !(flags & CRAVA_BATCH_NO_GRAPH);
  auto fail = [&](int code) { batch_free(b); return code; };
  for (int k = 0; k < n; ++k) {
    const crava_gpu_vintage &v = vin[k];
    crava_gpu_batch::Vintage w;
    w.ctx = v.ctx; w.in = v.in; w.out = v.out; w.precision = v.precision; w.nsim = v.nsim;
    w.seed = v.seed; w.first = v.first_index;
    if (v.nsim > 0) w.sim.assign(v.sim_out, v.sim_out + 3 * v.nsim);
    b->v.push_back(std::move(w));
    if (v.nsim > 0) {
      // the output table of the persistent realisation filter
      crava_gpu_batch::Vintage &bv = b->v.back();
      const size_t bytes = sizeof(float2 *) * 3 * (size_t)v.nsim;
      if (cudaMalloc(&bv.d_sim, bytes) != cudaSuccess) { bv.d_sim = nullptr; return fail(CRAVA_GPU_ERR_ALLOC); }
      if (cudaMemcpy(bv.d_sim, bv.sim.data(), bytes, cudaMemcpyHostToDevice) != cudaSuccess) return fail(CRAVA_GPU_ERR_CUDA);
    }
    bool seen = false;
    for (auto *c : b->ctxs) seen = seen || c == v.ctx;
    if (!seen) b->ctxs.push_back(v.ctx);
  }
  if (stream) {
    b->stream = static_cast<cudaStream_t>(stream);
  } else {
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) return fail(CRAVA_GPU_ERR_CUDA);
    b->own_stream = true;
  }
  for (size_t i = 0; i < b->ctxs.size(); ++i) {
    cudaStream_t s = nullptr;
    cudaEvent_t e = nullptr;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return fail(CRAVA_GPU_ERR_CUDA);
    b->cstream.push_back(s);
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return fail(CRAVA_GPU_ERR_CUDA);
    b->join.push_back(e);
  }
  if (cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) != cudaSuccess) return fail(CRAVA_GPU_ERR_CUDA);
  if (cudaMalloc(&b->epoch, sizeof(unsigned long long)) != cudaSuccess) return fail(CRAVA_GPU_ERR_ALLOC);
  if (cudaMemsetAsync(b->epoch, 0, sizeof(unsigned long long), b->stream) != cudaSuccess) return fail(CRAVA_GPU_ERR_CUDA);
  if (flags & CRAVA_BATCH_AUTOTUNE) {
    for (auto *c : b->ctxs) {
      for (auto &v : b->v)
        if (v.ctx == c) {
          if (cudaStreamSynchronize(b->stream) != cudaSuccess) return fail(CRAVA_GPU_ERR_CUDA);
          if ((rc = crava_gpu_autotune(c, &v.in, &v.out, v.precision, 2, nullptr))) return fail(rc);
          if (cudaStreamSynchronize(c->stream) != cudaSuccess) return fail(CRAVA_GPU_ERR_CUDA);
          break;
        }
    }
  }
  // warm-up run: workspaces, kernel attributes; realisations of epoch 0
  if ((rc = enqueue(b, false, false))) return fail(rc);
  if (cudaStreamSynchronize(b->stream) != cudaSuccess) return fail(CRAVA_GPU_ERR_CUDA);
  if (b->graph_mode) {
    const long long n0 = launches();
    cudaError_t e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) { set_last_error(e, "cudaStreamBeginCapture", __FILE__, __LINE__); return fail(CRAVA_GPU_ERR_CUDA); }
    rc = enqueue(b, true, true);
    cudaGraph_t g = nullptr;
    e = cudaStreamEndCapture(b->stream, &g);
    b->graph = g;
    const long long captured = launches() - n0;
    note_launch((int)-captured);  // recorded into the graph, not launched
    if (rc) return fail(rc);
    if (e != cudaSuccess) { set_last_error(e, "cudaStreamEndCapture", __FILE__, __LINE__); return fail(CRAVA_GPU_ERR_CUDA); }
    e = cudaGraphInstantiate(&b->exec, b->graph, 0);
    if (e != cudaSuccess) { set_last_error(e, "cudaGraphInstantiate", __FILE__, __LINE__); return fail(CRAVA_GPU_ERR_CUDA); }
    b->kernels = captured;
    e = cudaGraphUpload(b->exec, b->stream);
    if (e != cudaSuccess) { set_last_error(e, "cudaGraphUpload", __FILE__, __LINE__); return fail(CRAVA_GPU_ERR_CUDA); }
  }
  *out = b;
  return CRAVA_GPU_OK;
}

int crava_gpu_batch_run(crava_gpu_batch *b) {
  if (!b) return CRAVA_GPU_ERR_ARG;
  DeviceGuard guard(b->device);
  if (!b->graph_mode) return enqueue(b, false, true);
  CRAVA_CUDA_TRY(cudaGraphLaunch(b->exec, b->stream));
  note_launch((int)b->kernels);
  return CRAVA_GPU_OK;
}

int crava_gpu_batch_sync(crava_gpu_batch *b) {
  if (!b) return CRAVA_GPU_ERR_ARG;
  DeviceGuard guard(b->device);
  CRAVA_CUDA_TRY(cudaStreamSynchronize(b->stream));
  return CRAVA_GPU_OK;
}

int crava_gpu_batch_destroy(crava_gpu_batch *b) {
  batch_free(b);
  return CRAVA_GPU_OK;
}

}  // extern "C"
