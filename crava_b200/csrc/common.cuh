// common.cuh -- shared device helpers for the crava_b200 kernels (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "crava_gpu.h"

namespace crava {

// ---------------------------------------------------------------- launch count
void note_launch(int n = 1);
long long launches();

// ---------------------------------------------------------------- errors
#define CRAVA_CUDA_TRY(expr)                                  \
  do {                                                        \
    cudaError_t e_ = (expr);                                  \
    if (e_ != cudaSuccess) {                                  \
      ::crava::set_last_error(e_, #expr, __FILE__, __LINE__); \
      return CRAVA_GPU_ERR_CUDA;                              \
    }                                                         \
  } while (0)

#define CRAVA_LAUNCH_CHECK()                                                  \
  do {                                                                        \
    cudaError_t e_ = cudaGetLastError();                                      \
    if (e_ != cudaSuccess) {                                                  \
      ::crava::set_last_error(e_, "kernel launch", __FILE__, __LINE__);       \
      return CRAVA_GPU_ERR_CUDA;                                              \
    }                                                                         \
    ::crava::note_launch();                                                   \
  } while (0)

void set_last_error(cudaError_t e, const char *what, const char *file, int line);

// Raises fn's dynamic shared-memory limit to `bytes` on the current device
// when it is not already that high (one cudaFuncSetAttribute per kernel and
// size, so launches recorded into a CUDA graph make no attribute calls).
int func_smem(const void *fn, size_t bytes);

// ---------------------------------------------------------------- complex
struct __align__(8) cfloat { float x, y; };

__host__ __device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ float2 cmulc(float2 a, float2 b) {  // a * conj(b)
  return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__host__ __device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
__host__ __device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }

__host__ __device__ __forceinline__ double2 dadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ double2 dsub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ double2 dmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ double2 dmulc(double2 a, double2 b) {  // a * conj(b)
  return make_double2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}

// ---------------------------------------------------------------- grid geometry
struct Geom {
  int nxp, nyp, nzp;
  int cnxp, rnxp;
  long long csize, rsize;
  static Geom make(int nx, int ny, int nz) {
    Geom g;
    g.nxp = nx; g.nyp = ny; g.nzp = nz;
    g.cnxp = nx / 2 + 1; g.rnxp = 2 * g.cnxp;
    g.csize = (long long)g.cnxp * ny * nz;
    g.rsize = (long long)g.rnxp * ny * nz;
    return g;
  }
};

}  // namespace crava
