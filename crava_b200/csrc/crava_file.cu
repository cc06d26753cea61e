// crava_file.cu -- the reference's binary grid format on the device path.
//
// FFTGrid::writeCravaFile / readCravaFile (src/fftgrid.cpp:2399-2487): a
// text line "crava_fftgrid_binary", the simbox geometry (x0, y0, dx, dy as
// doubles, nx, ny as ints, IL0, XL0, ILStepX, ILStepY, XLStepX, XLStepY,
// angle as doubles), rnxp, nyp, nzp as ints, then the rsize floats of the
// padded real grid -- every number big-endian IEEE (NRLib::WriteBinary*,
// libs/nrlib/iotools/fileio.hpp:230-275, default END_BIG_ENDIAN).  The
// payload moves as raw bytes between the file, pinned host memory and HBM;
// the byte order is swapped on the device (one pass over the grid) instead
// of one call per float on the host.
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "context.cuh"

using namespace crava;

namespace {

constexpr int kThreads = 256;
const char kMagic[] = "crava_fftgrid_binary";

// Byte swap of n 4-byte words, src -> dst (may alias).
__global__ void __launch_bounds__(kThreads) k_bswap32(const uint32_t *src, uint32_t *dst, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = __byte_perm(src[i], 0, 0x0123);
}

void put_be(std::vector<unsigned char> &b, const void *p, int n) {
  const unsigned char *c = static_cast<const unsigned char *>(p);
  for (int i = n - 1; i >= 0; --i) b.push_back(c[i]);  // host is little-endian
}
template <typename T>
bool get_be(FILE *f, T *v) {
  unsigned char c[sizeof(T)], r[sizeof(T)];
  if (std::fread(c, 1, sizeof(T), f) != sizeof(T)) return false;
  for (size_t i = 0; i < sizeof(T); ++i) r[i] = c[sizeof(T) - 1 - i];
  std::memcpy(v, r, sizeof(T));
  return true;
}

int ensure_file_buffers(crava_gpu_ctx *c) {
  const size_t bytes = (size_t)c->g.rsize * sizeof(float);
  if (!c->file_host) {
    if (cudaMallocHost(&c->file_host, bytes) != cudaSuccess) { c->file_host = nullptr; return CRAVA_GPU_ERR_ALLOC; }
  }
  if (!c->file_dev) {
    if (cudaMalloc(&c->file_dev, bytes) != cudaSuccess) { c->file_dev = nullptr; return CRAVA_GPU_ERR_ALLOC; }
  }
  return CRAVA_GPU_OK;
}

}  // namespace

extern "C" {

int crava_gpu_crava_file_write(crava_gpu_ctx *c, const char *path, const float *grid,
                               const crava_gpu_grid_header *h) {
  if (!c || !path || !grid || !h) return CRAVA_GPU_ERR_ARG;
  DeviceGuard guard(c->device);
  int rc;
  if ((rc = ensure_file_buffers(c))) return rc;
  const long long n = c->g.rsize;
  k_bswap32<<<(unsigned)((n + kThreads - 1) / kThreads), kThreads, 0, c->stream>>>(
      reinterpret_cast<const uint32_t *>(grid), reinterpret_cast<uint32_t *>(c->file_dev), n);
  CRAVA_LAUNCH_CHECK();
  CRAVA_CUDA_TRY(cudaMemcpyAsync(c->file_host, c->file_dev, n * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  std::vector<unsigned char> hdr(kMagic, kMagic + sizeof(kMagic) - 1);
  hdr.push_back('\n');
  const double d0[4] = {h->x0, h->y0, h->dx, h->dy};
  for (double v : d0) put_be(hdr, &v, 8);
  put_be(hdr, &h->nx, 4);
  put_be(hdr, &h->ny, 4);
  const double d1[7] = {h->il0, h->xl0, h->il_step_x, h->il_step_y, h->xl_step_x, h->xl_step_y, h->angle};
  for (double v : d1) put_be(hdr, &v, 8);
  const int dims[3] = {c->g.rnxp, c->g.nyp, c->g.nzp};
  for (int v : dims) put_be(hdr, &v, 4);
  FILE *f = std::fopen(path, "wb");
  if (!f) return CRAVA_GPU_ERR_ARG;
  bool ok = std::fwrite(hdr.data(), 1, hdr.size(), f) == hdr.size();
  cudaError_t e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) { std::fclose(f); set_last_error(e, "crava file download", __FILE__, __LINE__); return CRAVA_GPU_ERR_CUDA; }
  ok = ok && std::fwrite(c->file_host, sizeof(float), (size_t)n, f) == (size_t)n;
  ok = (std::fclose(f) == 0) && ok;
  return ok ? CRAVA_GPU_OK : CRAVA_GPU_ERR_ARG;
}

int crava_gpu_crava_file_read(crava_gpu_ctx *c, const char *path, float *grid,
                              crava_gpu_grid_header *h) {
  if (!c || !path || !grid) return CRAVA_GPU_ERR_ARG;
  DeviceGuard guard(c->device);
  int rc;
  if ((rc = ensure_file_buffers(c))) return rc;
  FILE *f = std::fopen(path, "rb");
  if (!f) return CRAVA_GPU_ERR_ARG;
  char line[64];
  bool ok = std::fgets(line, sizeof line, f) != nullptr;  // getline: the type line
  crava_gpu_grid_header hh{};
  double d0[4], d1[7];
  int dims[3];
  for (int i = 0; ok && i < 4; ++i) ok = get_be(f, &d0[i]);
  ok = ok && get_be(f, &hh.nx) && get_be(f, &hh.ny);
  for (int i = 0; ok && i < 7; ++i) ok = get_be(f, &d1[i]);
  for (int i = 0; ok && i < 3; ++i) ok = get_be(f, &dims[i]);
  // the reference rejects a grid whose padded dimensions differ
  if (!ok || dims[0] != c->g.rnxp || dims[1] != c->g.nyp || dims[2] != c->g.nzp) {
    std::fclose(f);
    return CRAVA_GPU_ERR_ARG;
  }
  const long long n = c->g.rsize;
  ok = std::fread(c->file_host, sizeof(float), (size_t)n, f) == (size_t)n;
  std::fclose(f);
  if (!ok) return CRAVA_GPU_ERR_ARG;
  hh.x0 = d0[0]; hh.y0 = d0[1]; hh.dx = d0[2]; hh.dy = d0[3];
  hh.il0 = d1[0]; hh.xl0 = d1[1]; hh.il_step_x = d1[2]; hh.il_step_y = d1[3];
  hh.xl_step_x = d1[4]; hh.xl_step_y = d1[5]; hh.angle = d1[6];
  if (h) *h = hh;
  CRAVA_CUDA_TRY(cudaMemcpyAsync(c->file_dev, c->file_host, n * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  k_bswap32<<<(unsigned)((n + kThreads - 1) / kThreads), kThreads, 0, c->stream>>>(
      reinterpret_cast<const uint32_t *>(c->file_dev), reinterpret_cast<uint32_t *>(grid), n);
  CRAVA_LAUNCH_CHECK();
  // the staging buffer is reused by the next call: wait for the upload
  CRAVA_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return CRAVA_GPU_OK;
}

}  // extern "C"
