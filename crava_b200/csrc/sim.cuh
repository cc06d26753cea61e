// sim.cuh -- seeded noise spectra and the posterior Cholesky filter.
#pragma once

#include "common.cuh"
#include "solve.cuh"

namespace crava {

int noise_fill(const Geom &g, float2 *grid, uint64_t seed, uint64_t stream, cudaStream_t s);
int sim_filter(const Geom &g, const float2 *const cov[6], float2 *const seed[3],
               DevCounters *counters, cudaStream_t s);
// Noise for parameters p = 0,1,2 (streams stream0 + p) filtered in one pass.
int noise_filter(const Geom &g, const float2 *const cov[6], float2 *const out[3],
                 uint64_t seed, uint64_t stream0, DevCounters *counters, cudaStream_t s);

// nreal (<= 8) realisations in one pass: out[3 r + p], streams
// stream0 + 3 r + p, plus epoch_mul * (*epoch) when epoch (a device
// counter) is given.
int noise_filter_multi(const Geom &g, const float2 *const cov[6], float2 *const *out, int nreal,
                       uint64_t seed, uint64_t stream0, const unsigned long long *epoch,
                       unsigned long long epoch_mul, DevCounters *counters, cudaStream_t s);

// The realisation filter of several posteriors (the vintages of a batch,
// any grid sizes) in one persistent launch: a grid of the device's
// resident blocks walks the 256-bin blocks of every vintage in turn; per
// bin the posterior covariance is read and factorised once and applied to
// the noise of all the vintage's realisations.  Realisation r, parameter p
// of vintage v uses noise stream stream0 + 3 r + p + epoch_mul * (*epoch)
// (epoch optional), as noise_filter_multi does, so the values equal its
// batches of 8 bit for bit.
constexpr int kMaxSimVintages = 16;
struct SimVintage {
  const float2 *cov[6];
  float2 *const *out;  // device array of 3 nsim output spectra
  long long csize;
  int cnxp, nyp, nzp, nsim;
  uint64_t seed, stream0;
  unsigned long long epoch_mul;
  DevCounters *counters;
};
int noise_filter_vintages(const SimVintage *v, int nv, const unsigned long long *epoch, cudaStream_t s);

}  // namespace crava
