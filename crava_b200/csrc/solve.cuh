// solve.cuh -- per-kz operator tables and the per-bin posterior solve.
#pragma once

#include "common.cuh"

namespace crava {

// Device-resident per-kz tables of one context (see kz_tables_build).
struct KzTables {
  float2 *wd = nullptr;  // [nzp][nt]  D(k) * conj-wavelet: K = diag(wd) A
  float2 *e1 = nullptr;  // [nzp][nt]  errMult1
  float2 *e2 = nullptr;  // [nzp][nt]  errMult2
  float *e3 = nullptr;   // [nzp][nt]  errMult3
  int *inv = nullptr;    // [nzp]      invert_frequency
  int *order = nullptr;  // [nzp]      plane visiting order of the solve
                         //            (null: natural order)
  int *order_inv = nullptr;  // [n_inv]  the inverted planes alone (the
                             //          solve when the band-gated planes
                             //          were done by the forward z pass)
  int n_inv = -1;            // inverted planes (-1: order not built)
  // FP64 solve in the Woodbury form (woodbury.cuh): the per-plane tables
  // (sb::WbTable [nzp]) and room for the list of the blocks it defers
  // (defer_n = blocks of its grid, 128 bins per block); null: the form is
  // not used
  void *wb = nullptr;
  int *defer_list = nullptr;
  long long defer_n = 0;
};

// Constants of the solve, passed by value (kernel parameter space).
struct SolveConsts {
  int nt;
  float wnc;
  float A[CRAVA_GPU_MAX_THETA][3];
  double theta[CRAVA_GPU_MAX_THETA][CRAVA_GPU_MAX_THETA];
  double var0[6];  // (0,0) (1,1) (2,2) (0,1) (0,2) (1,2)
  // mixed form: a bin whose FP32 factor's condition bound exceeds this
  // takes one FP64 refinement step (0: every bin; a huge value: none)
  float kappa_refine;
  // launch shape of the FP64 / mixed solve (-1: the built-in choice of the
  // precision; 0-5: solve.cu)
  int solve_shape;
};

struct SolveGrids {
  float2 *mu[3];
  float2 *data[CRAVA_GPU_MAX_THETA];
  float2 *cov[6];
  const float2 *err;
};

struct DevCounters {
  unsigned long long chol_fail;
  unsigned long long nonfinite;
  unsigned long long refined;  // mixed form: bins that took the FP64 refinement step
  unsigned long long deferred; // FP64 Woodbury form: blocks left to the square-root kernel
};

// Default condition bound above which the mixed form refines a bin.
constexpr float kKappaRefineDefault = 1.0e4f;

int kz_tables_alloc(int nzp, int nt, KzTables *t);
// Fills t->order from t->inv (synchronises s): inverted (compute-heavy)
// and band-gated (memory-only) planes interleaved evenly, so the solve's
// blocks keep both the FP64 pipes and HBM busy.
// *n_inverted (optional) receives the number of inverted planes.
int kz_order_build(int nzp, KzTables *t, cudaStream_t s, int *n_inverted = nullptr);
void kz_tables_free(KzTables *t);
// Allocates the Woodbury tables and the deferred-block list for a grid of
// `plane` bins per kz plane (the FP64 solve's default form).
int kz_woodbury_alloc(int nzp, long long plane, KzTables *t);
// Fills the Woodbury tables from the kz tables (one kernel on s; call after
// the tables change).
int kz_woodbury_build(const SolveConsts &c, int nzp, const KzTables &t, cudaStream_t s);
// Builds the tables from the wavelets on the device (params: host struct).
int kz_tables_build(const crava_gpu_params &p, KzTables *t, cudaStream_t s);

// Builds the tables from wavelets already in device memory (d_norm may be
// null); launches one kernel on s and allocates nothing.
int kz_tables_build_device(const crava_gpu_params &p, const float *d_wavelet,
                           const float *d_norm, KzTables *t, cudaStream_t s);

// Per-bin solve over csize bins; plane = cnxp * nyp bins per kz.
// gated_done (FP64 and mixed forms, with the order built): the band-gated
// planes already hold the prior covariance (the forward z pass's ZPrior
// rule, fft.cuh), so only the inverted planes are visited.
int posterior_solve(const SolveConsts &c, const KzTables &t, const SolveGrids &g,
                    long long csize, long long plane, int precision,
                    DevCounters *counters, cudaStream_t s, bool gated_done = false);
// Counts the bins flagged by ZPrior epilogues (nf_bits, nwords words, and
// nf_any) into counters->nonfinite and clears the flags; one block, which
// returns at once when nothing was flagged.
int gated_nonfinite_count(unsigned *nf_bits, long long nwords, unsigned *nf_any, DevCounters *counters,
                          cudaStream_t s);
// FP32 form with the reference's operation order (separate translation
// unit compiled without FMA contraction).
int posterior_solve_fp32ref(const SolveConsts &c, const KzTables &t,
                            const SolveGrids &g, long long csize, long long plane,
                            DevCounters *counters, cudaStream_t s);

}  // namespace crava
