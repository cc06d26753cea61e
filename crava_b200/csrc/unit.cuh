// unit.cuh -- the fused posterior unit: xy-plane transforms with a
// thread-block cluster, and one kernel doing the z transform, the per-bin
// solve and the inverse z transform.
#pragma once

#include "fft.cuh"
#include "solve.cuh"

namespace crava {

constexpr int kMaxUnitGrids = 10 + CRAVA_GPU_MAX_THETA;

// Geometry of the plane kernels and of the column-pair workspace layout.
//   W grid: tile (ky, pair) holds the two columns kx = 2 pair, 2 pair + 1
//   for every z: float2 index ((ky * NP + pair) * nzp + z) * 2 + (kx & 1).
struct UnitPlan {
  Geom g;
  int hx;       // x line length: nxp/2 (even nxp) or nxp (odd)
  int even;
  int NP;       // column pairs = ceil(cnxp / 2)
  int CS;       // cluster size of the plane kernels (1, 2, 4 or 8)
  int R;        // rows per CTA = ceil(nyp / CS)
  int PP;       // pairs per CTA = ceil(NP / CS)
  int PR, PC;   // odd shared-memory pitches of the row band and the columns
  int SA, SB, SC;  // float2 per shared buffer
  size_t plane_smem;
  int zgroup;   // grids per z-transform group
  size_t z_smem;
  long long wgrid;  // float2 per workspace grid = nyp * NP * 2 * nzp
  bool ok;          // false: the fused path does not fit; use the 3-pass path
};

bool unit_plan(const Geom &g, int ntheta, UnitPlan *p);

// Forward transforms of n grids: real (reference layout) -> W layout.
int unit_plane_forward(const UnitPlan &p, const FftPlans &f, const float *const *src,
                       float2 *const *w, const float *scale, int n, cudaStream_t s);
// Inverse transforms of n grids: W layout -> real (reference layout), + addend.
int unit_plane_inverse(const UnitPlan &p, const FftPlans &f, const float2 *const *w,
                       float *const *dst, const float *scale, const float *const *addend,
                       int n, cudaStream_t s);
// z transform + solve + inverse z transform on the W grids (mu 3, data nt,
// cov 6, err 1), in place; err stays z-transformed.
int unit_zsolve(const UnitPlan &p, const FftPlans &f, const SolveConsts &c, const KzTables &t,
                float2 *const *w, int precision, DevCounters *counters, cudaStream_t s);

}  // namespace crava
