// interp.cu -- low-energy traces of a data grid filled from their
// neighbours, then the padding extrapolated from the edge traces.
//
// Replaces FFTGrid::interpolateSeismic (src/fftgrid.cpp:2564-2654) with
// interpolateTrace (:2658-2695) and extrapolateSeismic (:2699-2731), the
// step that closes Crava::divideDataByScaleWavelet (src/crava.cpp:690).
//
// The walk over the trace flags depends only on which traces are bad, not
// on their values, so it runs on the host over the energy map and emits
// the reference's exact sequence of trace interpolations; the device
// computes the energies (float sums in the reference's order), replays the
// interpolations in that order (one block, one trace at a time: a later
// interpolation may read an earlier one's result) and extrapolates the
// padding, whose sources lie inside the box of good traces and are never
// written by it, so that pass is fully parallel.
#include <math.h>

#include <vector>

#include "context.cuh"

using namespace crava;

namespace {

constexpr int kThreads = 256;

struct InterpArgs {
  float *grid;
  int nx, ny, nz, nxp, nyp, nzp, rnxp;
};

// Energy of each simbox trace over its nz samples, summed in k order.
__global__ void __launch_bounds__(kThreads) k_trace_energy(const __grid_constant__ InterpArgs a, float *energy) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.nx * a.ny) return;
  const int i = t % a.nx, j = t / a.nx;
  const long long plane = (long long)a.rnxp * a.nyp;
  const float *g = a.grid + i + (long long)a.rnxp * j;
  float e = 0.0f;
  for (int k = 0; k < a.nz; ++k) {
    const float v = g[k * plane];
    e = __fadd_rn(e, __fmul_rn(v, v));
  }
  energy[t] = e;
}

// One interpolation: the mean of the listed neighbours, written over the
// whole padded trace (interpolateTrace).
struct Op {
  int i, j, mask, nt;  // mask bits: left, right, up, down
};

__global__ void __launch_bounds__(kThreads) k_interp_ops(const __grid_constant__ InterpArgs a, const Op *ops,
                                                        int nops) {
  const long long plane = (long long)a.rnxp * a.nyp;
  for (int o = 0; o < nops; ++o) {
    const Op op = ops[o];
    float *g = a.grid + op.i + (long long)a.rnxp * op.j;
    for (int k = threadIdx.x; k < a.nzp; k += blockDim.x) {
      const long long kk = k * plane;
      float m = (op.mask & 1) ? g[kk - 1] : 0.0f;
      if (op.mask & 2) m = __fadd_rn(m, g[kk + 1]);
      if (op.mask & 4) m = __fadd_rn(m, g[kk - a.rnxp]);
      if (op.mask & 8) m = __fadd_rn(m, g[kk + a.rnxp]);
      g[kk] = __fdiv_rn(m, (float)op.nt);
    }
    __syncthreads();  // the next interpolation may read this trace
  }
}

// FFTGrid::getFillNumber (src/fftgrid.cpp:1319-1357) for i < np.
__device__ __forceinline__ int fill_number(int i, int n, int np) {
  if (i < n) return i;
  const int below = np - i - 1, above = i - n + 1;
  return above < below ? max(n - above, n / 2) : min(below, n / 2);
}

// FFTGrid::getDistToBoundary (src/fftgrid.cpp:1374-1414) for i < np.
__device__ __forceinline__ float dist_to_boundary(int i, int n, int np) {
  if (i < n) return 0.0f;
  const float taper = (float)((double)min(n, np - n) / 2.1);
  const int below = np - i, above = i - (n - 1);
  return above < below ? __fdiv_rn((float)above, taper) : __fdiv_rn((float)below, taper);
}

struct ExtrapArgs {
  InterpArgs g;
  int imin, imax, jmin, jmax;
};

// extrapolateSeismic: every padded cell outside the box of good traces
// takes its clamped fill trace's value times the cube of the taper.
__global__ void __launch_bounds__(kThreads) k_extrapolate(const __grid_constant__ ExtrapArgs e) {
  const InterpArgs &a = e.g;
  const long long n = (long long)a.nxp * a.nyp * a.nzp;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n) return;
  const int i = (int)(idx % a.nxp);
  const long long jk = idx / a.nxp;
  const int j = (int)(jk % a.nyp), k = (int)(jk / a.nyp);
  if (!(i < e.imin || i > e.imax || j < e.jmin || j > e.jmax)) return;
  const int refi = min(max(fill_number(i, a.nx, a.nxp), e.imin), e.imax);
  const int refj = min(max(fill_number(j, a.ny, a.nyp), e.jmin), e.jmax);
  const long long plane = (long long)a.rnxp * a.nyp;
  const float value = a.grid[refi + (long long)a.rnxp * refj + k * plane];
  const float dx = dist_to_boundary(i, a.nx, a.nxp), dy = dist_to_boundary(j, a.ny, a.nyp);
  const float dz = dist_to_boundary(k, a.nz, a.nzp);
  const double b = 1.0 - (double)__fmul_rn(dx, dx) - (double)__fmul_rn(dy, dy) - (double)__fmul_rn(dz, dz);
  const float mult = (float)pow(fmax(b, 0.0), 3.0);
  a.grid[i + (long long)a.rnxp * j + k * plane] = __fmul_rn(mult, value);
}

// The flag walk of interpolateSeismic (src/fftgrid.cpp:2589-2650) on the
// host: the ordered interpolations interpolateTrace would make.
struct Walk {
  int nx, ny;
  std::vector<short> flags;
  std::vector<Op> ops;

  // interpolateTrace without the arithmetic: records the interpolation
  // when at least two neighbours are good, and returns the flag.
  int trace(int index, int i, int j) {
    const bool left = i > 0 && (flags[index - 1] % 2) == 0;
    const bool right = i < nx - 1 && (flags[index + 1] % 2) == 0;
    const bool up = j > 0 && (flags[index - nx] % 2) == 0;
    const bool down = j < ny - 1 && (flags[index + nx] % 2) == 0;
    const int nt = (int)left + (int)right + (int)up + (int)down;
    if (nt > 1) {
      ops.push_back(Op{i, j, (left ? 1 : 0) | (right ? 2 : 0) | (up ? 4 : 0) | (down ? 8 : 0), nt});
      flags[index]--;
    }
    return flags[index];
  }
};

}  // namespace

extern "C" int crava_gpu_interpolate_seismic(crava_gpu_ctx *c, float *grid, int nx, int ny,
                                             float energy_threshold, int *n_interpolated,
                                             int *n_zero) {
  if (!c || !grid || (reinterpret_cast<uintptr_t>(grid) & 7u)) return CRAVA_GPU_ERR_ARG;
  const Geom &g = c->g;
  if (nx < 1 || ny < 1 || nx > g.nxp || ny > g.nyp || c->p.nz < 1 || c->p.nz > g.nzp) return CRAVA_GPU_ERR_ARG;
  if (!isfinite(energy_threshold)) return CRAVA_GPU_ERR_ARG;
  DeviceGuard guard(c->device);
  const cudaStream_t s = c->stream;
  InterpArgs a{grid, nx, ny, c->p.nz, g.nxp, g.nyp, g.nzp, g.rnxp};
  const int ntr = nx * ny;
  float *d_energy = nullptr;
  Op *d_ops = nullptr;
  int rc = CRAVA_GPU_OK;
  std::vector<float> energy(ntr);
  auto run = [&]() -> int {
    CRAVA_CUDA_TRY(cudaMalloc(&d_energy, sizeof(float) * ntr));
    k_trace_energy<<<(ntr + kThreads - 1) / kThreads, kThreads, 0, s>>>(a, d_energy);
    CRAVA_LAUNCH_CHECK();
    CRAVA_CUDA_TRY(cudaMemcpyAsync(energy.data(), d_energy, sizeof(float) * ntr, cudaMemcpyDeviceToHost, s));
    CRAVA_CUDA_TRY(cudaStreamSynchronize(s));
    // flags: bit 0 this trace bad, bit 1 a previous trace bad
    float total = 0.0f;
    for (int t = 0; t < ntr; ++t) total += energy[t];
    const float limit = energy_threshold * total / (float)(nx * ny);
    Walk w{nx, ny, std::vector<short>(ntr), {}};
    int flag = 0, imin = nx, imax = 0, jmin = ny, jmax = 0, ninter = 0, ninter0 = 0;
    for (int j = 0, index = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i, ++index) {
        int cur = 0;
        if (energy[index] <= limit) {
          cur = 1;
          ++ninter;
          if (energy[index] == 0.0f) ++ninter0;
        }
        w.flags[index] = (short)(flag + cur);
        if (cur == 1) {
          flag = 2;
        } else {
          imin = std::min(imin, i); imax = std::max(imax, i);
          jmin = std::min(jmin, j); jmax = std::max(jmax, j);
        }
      }
    for (int j = 0, cur = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i, ++cur) {
        if ((w.flags[cur] % 2) != 1) continue;
        if ((w.trace(cur, i, j) % 2) != 0) continue;
        int index = cur - 1;
        while (index >= 0 && w.flags[index] > 1) {
          if ((w.flags[index] % 2) == 1) w.trace(index, index % nx, index / nx);
          index--;
        }
        if (index < 0) index = 0;
        index++;
        while (index <= cur && w.flags[index - 1] == 0) {
          if (w.flags[index] > 1) w.flags[index] -= 2;
          index++;
        }
      }
    if (n_interpolated) *n_interpolated = ninter;
    if (n_zero) *n_zero = ninter0;
    if (!w.ops.empty()) {
      CRAVA_CUDA_TRY(cudaMalloc(&d_ops, sizeof(Op) * w.ops.size()));
      CRAVA_CUDA_TRY(cudaMemcpyAsync(d_ops, w.ops.data(), sizeof(Op) * w.ops.size(), cudaMemcpyHostToDevice, s));
      k_interp_ops<<<1, kThreads, 0, s>>>(a, d_ops, (int)w.ops.size());
      CRAVA_LAUNCH_CHECK();
    }
    // with no good trace at all there is no box to extrapolate from
    if (imin <= imax && jmin <= jmax) {
      ExtrapArgs e{a, imin, imax, jmin, jmax};
      const long long n = (long long)g.nxp * g.nyp * g.nzp;
      k_extrapolate<<<(unsigned)((n + kThreads - 1) / kThreads), kThreads, 0, s>>>(e);
      CRAVA_LAUNCH_CHECK();
    }
    CRAVA_CUDA_TRY(cudaStreamSynchronize(s));
    return CRAVA_GPU_OK;
  };
  rc = run();
  cudaFree(d_energy);
  cudaFree(d_ops);
  return rc;
}
