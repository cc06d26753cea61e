// Drives CravaDevice / FFTGridDevice (crava_b200/host/crava_device.hpp) the
// way Crava::Crava drives FFTGrid: forward transforms of the means and
// stacks, computePostMeanResidAndFFTCov, inverse transforms of residuals and
// covariances.  Reads raw float32 grids and parameters from a directory
// written by tests/test_host_mirror.py and writes the outputs back there.
//
// With a second argument "cursor" the grids are filled through the
// element cursors (setAccessMode(WRITE) + setNextReal, as
// FFTGrid::fillInFromArray does, src/fftgrid.cpp:940-990), the posterior
// spectra are walked with getNextComplex in the order of the reference's
// per-bin loop (src/crava.cpp:1085-1150) and compared with the bulk
// download, a READANDWRITE pass writes every value back through
// setNextComplex, and the real outputs are read with getNextReal.
// Prints "cursor_mismatch N" (N values that differ bit for bit).
#include <cstdio>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "crava_device.hpp"

using crava_b200::FFTGridDevice;

static std::vector<char> slurp(const std::string &path) {
  std::ifstream f(path, std::ios::binary);
  return std::vector<char>((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
}

int main(int argc, char **argv) {
  if (argc < 2) { std::fprintf(stderr, "usage: %s dir\n", argv[0]); return 2; }
  const std::string dir = argv[1];
  const bool cursor = argc > 2 && std::string(argv[2]) == "cursor";
  long long mismatch = 0;
  std::vector<char> hdr = slurp(dir + "/dims.bin");
  const int *dims = reinterpret_cast<const int *>(hdr.data());
  const int nx = dims[0], ny = dims[1], nz = dims[2], nt = dims[3], prec = dims[4];
  std::vector<char> wav = slurp(dir + "/wavelet.bin"), A = slurp(dir + "/A.bin");
  std::vector<char> th = slurp(dir + "/theta.bin"), v0 = slurp(dir + "/var0.bin");
  std::vector<char> sc = slurp(dir + "/scalars.bin");
  const double *s = reinterpret_cast<const double *>(sc.data());
  crava_gpu_params p{};
  p.nxp = nx; p.nyp = ny; p.nzp = nz; p.ntheta = nt; p.nz = (int)s[0]; p.precision = prec;
  p.lz = s[1]; p.min_rel_thick = s[2]; p.low_cut = (float)s[3]; p.high_cut = (float)s[4];
  p.wnc = (float)s[5];
  p.wavelet = reinterpret_cast<const float *>(wav.data());
  p.A = reinterpret_cast<const float *>(A.data());
  p.theta_cov = reinterpret_cast<const double *>(th.data());
  p.var0 = reinterpret_cast<const double *>(v0.data());
  try {
    crava_b200::CravaDevice crava(p);
    auto load = [&](const std::string &name, int type) {
      auto *g = crava.createFFTGrid(nx, ny, nz, type);
      std::vector<char> b = slurp(dir + "/" + name + ".bin");
      const float *v = reinterpret_cast<const float *>(b.data());
      if (cursor) {
        g->setAccessMode(FFTGridDevice::WRITE);
        for (long long i = 0; i < g->getrsize(); ++i) g->setNextReal(v[i]);
        g->endAccess();
      } else {
        g->upload(v);
      }
      return g;
    };
    // the spectra of a transformed grid through getNextComplex, bin by bin
    // in the reference loop's order, against the bulk download
    auto walk_complex = [&](FFTGridDevice *g) {
      std::vector<float> bulk((size_t)g->getrsize());
      g->download(bulk.data());
      g->setAccessMode(FFTGridDevice::READ);
      const int cnx = g->getCNxp();
      for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
          for (int i = 0; i < cnx; ++i) {
            const crava_b200::fftw_complex c = g->getNextComplex();
            const size_t o = 2 * ((size_t)i + (size_t)cnx * (j + (size_t)ny * k));
            if (std::memcmp(&c.re, &bulk[o], 4) || std::memcmp(&c.im, &bulk[o + 1], 4)) ++mismatch;
          }
      if (g->getCounterForGet() != 0) ++mismatch;  // the cursor wrapped to the start
      g->endAccess();
      // read-and-write pass: every value written back unchanged
      g->setAccessMode(FFTGridDevice::READANDWRITE);
      for (long long b = 0; b < g->getcsize(); ++b) g->setNextComplex(g->getNextComplex());
      g->endAccess();
      std::vector<float> again((size_t)g->getrsize());
      g->download(again.data());
      for (size_t o = 0; o < again.size(); ++o)
        if (std::memcmp(&again[o], &bulk[o], 4)) ++mismatch;
    };
    FFTGridDevice *mu[3], *cov[6];
    std::vector<FFTGridDevice *> data(nt);
    for (int q = 0; q < 3; ++q) mu[q] = load("mu" + std::to_string(q), FFTGridDevice::PARAMETER);
    for (int l = 0; l < nt; ++l) data[l] = load("data" + std::to_string(l), FFTGridDevice::DATA);
    for (int t = 0; t < 6; ++t) cov[t] = load("cov" + std::to_string(t), FFTGridDevice::COVARIANCE);
    FFTGridDevice *err = load("err", FFTGridDevice::COVARIANCE);
    for (auto *g : data) g->fftInPlace();   // src/crava.cpp:175-179
    for (auto *g : mu) g->fftInPlace();     // src/crava.cpp:188-190
    crava.computePostMeanResidAndFFTCov(mu, data.data(), cov, err, prec);
    if (cursor) {
      for (auto *g : data) walk_complex(g);  // residual spectra
      for (auto *g : cov) walk_complex(g);   // posterior covariance spectra
    }
    for (auto *g : data) g->invFFTInPlace();  // residuals (src/crava.cpp:1189-1206)
    for (auto *g : cov) g->invFFTInPlace();   // invFFTCovGrids (src/crava.cpp:218)
    std::vector<float> buf((size_t)2 * (nx / 2 + 1) * ny * nz);
    auto save = [&](FFTGridDevice *g, const std::string &name) {
      g->download(buf.data());
      if (cursor) {
        g->setAccessMode(FFTGridDevice::READ);
        for (size_t i = 0; i < buf.size(); ++i) {
          const float v = g->getNextReal();
          if (std::memcmp(&v, &buf[i], 4)) ++mismatch;
        }
        g->endAccess();
      }
      std::ofstream f(dir + "/out_" + name + ".bin", std::ios::binary);
      f.write(reinterpret_cast<const char *>(buf.data()), buf.size() * sizeof(float));
    };
    for (int q = 0; q < 3; ++q) save(mu[q], "mu" + std::to_string(q));
    for (int l = 0; l < nt; ++l) save(data[l], "data" + std::to_string(l));
    for (int t = 0; t < 6; ++t) save(cov[t], "cov" + std::to_string(t));
    crava_gpu_stats st = crava.stats();
    std::printf("chol_fail_bins %lld nonfinite_bins %lld\n", st.chol_fail_bins, st.nonfinite_bins);
    if (cursor) std::printf("cursor_mismatch %lld\n", mismatch);
    for (auto *g : mu) delete g;
    for (auto *g : data) delete g;
    for (auto *g : cov) delete g;
    delete err;
  } catch (const crava_b200::Error &e) {
    std::fprintf(stderr, "error: %s\n", e.what());
    return 1;
  }
  return 0;
}
