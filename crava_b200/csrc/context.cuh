// context.cuh -- the state behind the C ABI's crava_gpu_ctx handle and the
// internal steps that the entry points compose (capi.cu, batch.cu).
#pragma once

#include <vector>

#include "common.cuh"
#include "fft.cuh"
#include "sim.cuh"
#include "solve.cuh"
#include "unit.cuh"

struct crava_gpu_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  crava_gpu_params p{};
  std::vector<float> wavelet, wnorm, A;
  std::vector<double> theta, var0;
  crava::Geom g{};
  crava::FftPlans plans{};
  crava::KzTables tables{};
  crava::SolveConsts consts{};
  crava::DevCounters *counters = nullptr;  // device
  cudaEvent_t ev[4] = {};           // start, after forward, after solve, end
  bool timed = false;               // events of the last call are valid
  // fused unit (plane kernels + z/solve kernel) and its workspace
  crava::UnitPlan uplan{};
  bool fused = false;  // the pass-by-pass path is faster; set_fused(1) selects the fused unit kernels
  float2 *W = nullptr;  // (10 + ntheta) grids in the column-pair layout
  // per-kernel profiling (events around each launch when enabled)
  bool prof = false;
  struct Rec { int kind; cudaEvent_t a, b; double bytes; };
  std::vector<Rec> recs;
  std::vector<cudaEvent_t> pool;
  double prof_ms[16] = {};
  double prof_bytes[16] = {};
  long long prof_n[16] = {};
  // host-buffer path
  float *work = nullptr;  // (10 + ntheta) grids per slot, 1 or 2 slots
  int work_slots = 0;
  cudaStream_t s_in = nullptr, s_out = nullptr;
  std::vector<cudaEvent_t> grid_ev;
  cudaEvent_t slot_done[2] = {};  // last download of a slot's step
  long long host_seq = 0;          // asynchronous host steps enqueued
  // set while a batch captures this context's work into a CUDA graph: the
  // stage-timing events are not recorded (they would become graph nodes)
  bool capture = false;
  // synthetic seismic: per-angle spectral filters [ntheta][nzp] (device)
  float2 *synt_H = nullptr;
  // independent transforms of a unit run on `lanes` streams (1: the
  // context's stream only), forked from and joined back to it
  static constexpr int kMaxLanes = 4;
  // (measured per 256x256x512x5 unit: 6.08 / 5.44 / 5.40 / 5.47 ms with
  // 1 / 2 / 3 / 4 lanes)
  int lanes = 3;
  cudaStream_t lane_s[kMaxLanes] = {};
  cudaEvent_t lane_fork = nullptr, lane_join[kMaxLanes] = {};
  // .crava file staging: pinned host and device buffers of one grid
  float *file_host = nullptr;
  float *file_dev = nullptr;
  // inverted kz planes (band flag set): the solve moves every spectrum of
  // their bins and only the covariance spectra of the others
  int n_inverted = 0;
  // prior fills: lateral [nyp][nxp] then temporal [nzp] correlation (device)
  float *prior_buf = nullptr;
  // divideDataByScaleWavelet scratch (tables, per-trace values, row
  // padding), kept between calls and grown when a call needs more
  char *div_buf = nullptr;
  size_t div_bytes = 0;
  // log marginal likelihood: device operator table, per-block partial sums
  // and failure count, and their pinned host copy, kept between calls
  char *ll_buf = nullptr;
  size_t ll_bytes = 0;
  char *ll_host = nullptr;
  size_t ll_host_bytes = 0;
  // bins whose band-gated prior (written by the forward z pass) is not
  // finite: one bit per bin, then the any-flag word (allocated and zeroed
  // with the context; the counting kernel clears what it counts)
  unsigned *gated_nf = nullptr;
  long long gated_nf_words = 0;
};

namespace crava {

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) == cudaSuccess && prev != dev) cudaSetDevice(dev);
    else prev = -1;
  }
  ~DeviceGuard() { if (prev >= 0) cudaSetDevice(prev); }
};

int check_grids(const crava_gpu_ctx *c, const crava_gpu_grids *gr);
int valid_precision(int prec);
bool use_fused(const crava_gpu_ctx *c, int precision);
// Forward transform of one grid, src -> dst (src == dst: in place); zp
// (optional): the band-gated covariance rule in the z pass's store.
int pass_forward(crava_gpu_ctx *c, const float *src, float *dst, int type, const ZPrior *zp = nullptr);
// Inverse transform in place; addend (optional) is added to the real output.
int pass_inverse(crava_gpu_ctx *c, float *grid, int type, const float *addend = nullptr);
// gated_done: the forward z passes applied the band-gated rule (the
// zp of gated_prior_setup) to the six covariance grids.
int pass_solve(crava_gpu_ctx *c, const crava_gpu_grids *gr, int precision, bool gated_done = false);
// Whether the unit's forward z passes can take over the band-gated bins of
// the solve (FP64 and mixed forms, z passes that have the rule, the plane
// order built, the flags allocated with the context); if so fills zp[6]
// (cov grids in unit order).  Allocates nothing.
int gated_prior_setup(crava_gpu_ctx *c, int precision, ZPrior zp[6], bool *on);
// After the forward passes that took zp: the flagged bins into the counters.
int gated_prior_count(crava_gpu_ctx *c);
// Transforms, solve and inverse transforms (in == out: in place).
int run_unit(crava_gpu_ctx *c, const crava_gpu_grids *in, const crava_gpu_grids *out,
             int precision);
// Records stage event i on the context's stream (skipped during capture).
int stage_event(crava_gpu_ctx *c, int i);
// Inverse transforms of n realisation grids (parameter p = k % 3 of grid
// k) with post_mean[p] added, spread over the context's transform lanes.
int inverse_realisations(crava_gpu_ctx *c, float *const *grids, int n, const float *const post_mean[3]);
// count realisations from the posterior covariance spectra cv: realisation
// r uses noise streams 3 (first + r) + p, plus 3 epoch_stride (*epoch) when
// epoch is given (a device counter), and gets post_mean added.
int simulate_batches(crava_gpu_ctx *c, const float2 *const cv[6], const float *const post_mean[3],
                     uint64_t seed, uint64_t first, int count, float *const *out,
                     const unsigned long long *epoch, unsigned long long epoch_stride);

// Every simbox trace of each grid[l] multiplied by the conjugate of its
// local wavelet's spectrum getCAmp(k, relThick) (with local shift / gain),
// divided by pre_div before and post_div after the transforms; the grids
// are spectra when inverse_first (transformed back first).  (divide.cu)
int multiply_local_wavelet(crava_gpu_ctx *c, float *const *grids, const double *rel_thick, int nx, int ny,
                           float dz, const float *shift, const float *gain, float pre_div, float post_div,
                           bool inverse_first);

}  // namespace crava
