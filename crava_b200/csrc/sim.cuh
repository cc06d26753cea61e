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

}  // namespace crava
