// crava_device.hpp -- C++ host classes over the C ABI (include/crava_gpu.h),
// mirroring the reference interfaces this library replaces:
//
//   FFTGridDevice  the device counterpart of FFTGrid (src/fftgrid.h): one
//                  padded grid in HBM, the same grid types and the same
//                  fftInPlace / invFFTInPlace scalings;
//   CravaDevice    the hot path of Crava (src/crava.h):
//                  computePostMeanResidAndFFTCov and simulate.
//
// Header only; link with crava_b200/lib/libcrava_gpu.so and the CUDA
// runtime.  Errors throw crava_b200::Error carrying the ABI status.
#pragma once

#include <cuda_runtime.h>

#include <stdexcept>
#include <string>
#include <vector>

#include "crava_gpu.h"

namespace crava_b200 {

class Error : public std::runtime_error {
 public:
  Error(const std::string &what, int status)
      : std::runtime_error(what + ": " + crava_gpu_status_string(status)), status_(status) {}
  int status() const { return status_; }

 private:
  int status_;
};

inline void check(int status, const char *what) {
  if (status != CRAVA_GPU_OK) throw Error(what, status);
}

// FFTW 2.1.2's complex element (libs/fft/include/fftw.h:58): what the
// reference's getNextComplex / setNextComplex pass.
struct fftw_complex {
  float re, im;
};

// A padded grid resident in HBM (layout of src/fftgrid.cpp:37-67).
//
// The reference reads and writes grids element by element through stateful
// cursors (getNextReal / setNextReal / getNextComplex / setNextComplex,
// src/fftgrid.cpp:1418-1431, 1603-1617) bracketed by setAccessMode /
// endAccess (src/fftgrid.h:168-173; FFTFileGrid, src/fftfilegrid.cpp:104-150,
// is the precedent for a grid whose values live elsewhere).  Here the values
// live in HBM, so the cursors work on a host mirror: setAccessMode(READ,
// READANDWRITE or RANDOMACCESS) downloads the grid into the mirror,
// endAccess() uploads it back after WRITE, READANDWRITE or a modified
// RANDOMACCESS, and the cursors walk the mirror in the reference's linear
// order (x fastest, then y, then z; rnxp reals or cnxp complex per row),
// wrapping to the start after the last element as the reference does.
// Copies are ordered on `stream` (the stream of the context's work) and
// wait for that stream only.
class FFTGridDevice {
 public:
  // FFTGrid::gridTypes (src/fftgrid.h:172)
  enum gridTypes { CTMISSING, DATA, PARAMETER, COVARIANCE };
  // FFTGrid::accessMode (src/fftgrid.h:168)
  enum accessMode { NONE, READ, WRITE, READANDWRITE, RANDOMACCESS };

  FFTGridDevice(crava_gpu_ctx *ctx, int nxp, int nyp, int nzp, int type = PARAMETER,
                cudaStream_t stream = nullptr)
      : ctx_(ctx), nxp_(nxp), nyp_(nyp), nzp_(nzp), type_(type), stream_(stream) {
    cnxp_ = nxp / 2 + 1;
    rnxp_ = 2 * cnxp_;
    rsize_ = (long long)rnxp_ * nyp * nzp;
    csize_ = (long long)cnxp_ * nyp * nzp;
    if (cudaMalloc(&data_, sizeof(float) * rsize_) != cudaSuccess) throw Error("FFTGridDevice", CRAVA_GPU_ERR_ALLOC);
  }
  ~FFTGridDevice() { cudaFree(data_); }
  FFTGridDevice(const FFTGridDevice &) = delete;
  FFTGridDevice &operator=(const FFTGridDevice &) = delete;

  void setType(int t) { type_ = t; }
  int getType() const { return type_; }
  bool getIsTransformed() const { return transformed_; }
  void setTransformedStatus(bool s) { transformed_ = s; }
  int getNxp() const { return nxp_; }
  int getNyp() const { return nyp_; }
  int getNzp() const { return nzp_; }
  int getCNxp() const { return cnxp_; }
  int getRNxp() const { return rnxp_; }
  long long getcsize() const { return csize_; }
  long long getrsize() const { return rsize_; }
  float *devicePtr() { return data_; }
  int getCounterForGet() const { return (int)get_; }
  int getCounterForSet() const { return (int)set_; }

  // FFTGrid::fftInPlace (src/fftgrid.cpp:1803-1829)
  void fftInPlace() {
    if (transformed_) throw Error("fftInPlace on a transformed grid", CRAVA_GPU_ERR_STATE);
    if (mode_ != NONE) throw Error("fftInPlace during an access", CRAVA_GPU_ERR_STATE);
    check(crava_gpu_fft_r2c(ctx_, data_, type_), "fftInPlace");
    transformed_ = true;
  }
  // FFTGrid::invFFTInPlace (src/fftgrid.cpp:1831-1862)
  void invFFTInPlace() {
    if (!transformed_) throw Error("invFFTInPlace on a real grid", CRAVA_GPU_ERR_STATE);
    if (mode_ != NONE) throw Error("invFFTInPlace during an access", CRAVA_GPU_ERR_STATE);
    check(crava_gpu_fft_c2r(ctx_, data_, type_), "invFFTInPlace");
    transformed_ = false;
  }
  // Bulk replacements of the setNextReal / getNextReal cursors.
  void upload(const float *host, bool transformed = false) {
    if (cudaMemcpyAsync(data_, host, sizeof(float) * rsize_, cudaMemcpyHostToDevice, stream_) != cudaSuccess ||
        cudaStreamSynchronize(stream_) != cudaSuccess)
      throw Error("upload", CRAVA_GPU_ERR_CUDA);
    transformed_ = transformed;
  }
  void download(float *host) const {
    if (cudaMemcpyAsync(host, data_, sizeof(float) * rsize_, cudaMemcpyDeviceToHost, stream_) != cudaSuccess ||
        cudaStreamSynchronize(stream_) != cudaSuccess)
      throw Error("download", CRAVA_GPU_ERR_CUDA);
  }

  // FFTGrid::setAccessMode / endAccess (src/fftgrid.h:172-173)
  void setAccessMode(int mode) {
    if (mode_ != NONE) throw Error("setAccessMode: previous access not ended", CRAVA_GPU_ERR_STATE);
    if (mode < NONE || mode > RANDOMACCESS) throw Error("setAccessMode", CRAVA_GPU_ERR_ARG);
    if (mode != NONE) mirror_.resize((size_t)rsize_);
    if (mode == READ || mode == READANDWRITE || mode == RANDOMACCESS) download(mirror_.data());
    mode_ = mode;
    modified_ = false;
  }
  void endAccess() {
    if ((mode_ == WRITE || mode_ == READANDWRITE || (mode_ == RANDOMACCESS && modified_)))
      upload(mirror_.data(), transformed_);
    mode_ = NONE;
    get_ = set_ = 0;
  }

  // FFTGrid::getNextComplex / getNextReal (src/fftgrid.cpp:1418-1445)
  fftw_complex getNextComplex() {
    if (!transformed_ || (mode_ != READ && mode_ != READANDWRITE))
      throw Error("getNextComplex", CRAVA_GPU_ERR_STATE);
    const fftw_complex *c = reinterpret_cast<const fftw_complex *>(mirror_.data());
    const fftw_complex v = c[get_];
    if (++get_ == csize_) get_ = 0;
    return v;
  }
  float getNextReal() {
    if (transformed_ || (mode_ != READ && mode_ != READANDWRITE))
      throw Error("getNextReal", CRAVA_GPU_ERR_STATE);
    const float v = mirror_[(size_t)get_];
    if (++get_ == rsize_) get_ = 0;
    return v;
  }
  // FFTGrid::setNextComplex / setNextReal (src/fftgrid.cpp:1603-1650)
  int setNextComplex(fftw_complex v) {
    if (!transformed_ || (mode_ != WRITE && mode_ != READANDWRITE))
      throw Error("setNextComplex", CRAVA_GPU_ERR_STATE);
    reinterpret_cast<fftw_complex *>(mirror_.data())[set_] = v;
    if (++set_ == csize_) set_ = 0;
    return 0;
  }
  int setNextReal(float v) {
    if (transformed_ || (mode_ != WRITE && mode_ != READANDWRITE))
      throw Error("setNextReal", CRAVA_GPU_ERR_STATE);
    mirror_[(size_t)set_] = v;
    if (++set_ == rsize_) set_ = 0;
    return 0;
  }
  // FFTGrid::getRealValue / setRealValue / getComplexValue (RANDOMACCESS;
  // src/fftgrid.cpp:1460-1600), inside the padded grid only
  float getRealValue(int i, int j, int k) const {
    if (mode_ != RANDOMACCESS || transformed_) throw Error("getRealValue", CRAVA_GPU_ERR_STATE);
    return mirror_[(size_t)i + (size_t)rnxp_ * (j + (size_t)nyp_ * k)];
  }
  int setRealValue(int i, int j, int k, float v) {
    if (mode_ != RANDOMACCESS || transformed_) throw Error("setRealValue", CRAVA_GPU_ERR_STATE);
    mirror_[(size_t)i + (size_t)rnxp_ * (j + (size_t)nyp_ * k)] = v;
    modified_ = true;
    return 0;
  }
  fftw_complex getComplexValue(int i, int j, int k) const {
    if (mode_ != RANDOMACCESS || !transformed_) throw Error("getComplexValue", CRAVA_GPU_ERR_STATE);
    return reinterpret_cast<const fftw_complex *>(mirror_.data())[(size_t)i + (size_t)cnxp_ * (j + (size_t)nyp_ * k)];
  }

 private:
  crava_gpu_ctx *ctx_;
  int nxp_, nyp_, nzp_, cnxp_, rnxp_;
  long long rsize_, csize_;
  int type_;
  cudaStream_t stream_ = nullptr;
  bool transformed_ = false;
  float *data_ = nullptr;
  // cursor state (host mirror of the device values during an access)
  int mode_ = NONE;
  bool modified_ = false;
  long long get_ = 0, set_ = 0;
  std::vector<float> mirror_;
};

// The hot path of Crava on device grids.
class CravaDevice {
 public:
  CravaDevice(const crava_gpu_params &p, int device = 0, cudaStream_t stream = nullptr) : stream_(stream) {
    check(crava_gpu_create(&p, device, stream, &ctx_), "crava_gpu_create");
    nt_ = p.ntheta;
  }
  ~CravaDevice() { crava_gpu_destroy(ctx_); }
  CravaDevice(const CravaDevice &) = delete;
  CravaDevice &operator=(const CravaDevice &) = delete;

  crava_gpu_ctx *ctx() { return ctx_; }

  // Crava::createFFTGrid (src/crava.cpp:1829-1860): a grid of this
  // context's geometry whose copies run on the context's stream.  The
  // caller owns it (delete).
  FFTGridDevice *createFFTGrid(int nxp, int nyp, int nzp, int type = FFTGridDevice::PARAMETER) {
    return new FFTGridDevice(ctx_, nxp, nyp, nzp, type, stream_);
  }

  // Crava::computePostMeanResidAndFFTCov (src/crava.cpp:887-1295): means
  // and stacks arrive transformed (src/crava.cpp:175-190); the prior
  // covariances and the noise correlation are transformed here (:1003,
  // :1012); on return the means hold the real-domain posterior mean
  // (:1181-1183), the stacks the residual spectra and the covariances the
  // posterior covariance spectra.  Returns 0, as the reference does.
  int computePostMeanResidAndFFTCov(FFTGridDevice *mu[3], FFTGridDevice **data, FFTGridDevice *cov[6],
                                    FFTGridDevice *errCorr, int precision = CRAVA_SOLVE_MIXED) {
    for (int t = 0; t < 6; ++t)
      if (!cov[t]->getIsTransformed()) cov[t]->fftInPlace();
    if (!errCorr->getIsTransformed()) errCorr->fftInPlace();
    crava_gpu_grids g{};
    for (int q = 0; q < 3; ++q) g.mu[q] = mu[q]->devicePtr();
    for (int l = 0; l < nt_; ++l) g.data[l] = data[l]->devicePtr();
    for (int t = 0; t < 6; ++t) g.cov[t] = cov[t]->devicePtr();
    g.err_corr = errCorr->devicePtr();
    check(crava_gpu_posterior(ctx_, &g, precision), "computePostMeanResidAndFFTCov");
    for (int q = 0; q < 3; ++q) mu[q]->invFFTInPlace();
    return 0;
  }

  // Crava::simulate (src/crava.cpp:1415-1599) for `count` realisations:
  // out[3 r + p] receives parameter p of realisation r (real domain).
  int simulate(FFTGridDevice *postCov[6], FFTGridDevice *postMean[3], uint64_t seed, int firstIndex,
               std::vector<FFTGridDevice *> &out) {
    const float *cv[6];
    const float *pm[3];
    for (int t = 0; t < 6; ++t) cv[t] = postCov[t]->devicePtr();
    for (int p = 0; p < 3; ++p) pm[p] = postMean[p]->devicePtr();
    std::vector<float *> o(out.size());
    for (size_t i = 0; i < out.size(); ++i) o[i] = out[i]->devicePtr();
    check(crava_gpu_simulate(ctx_, cv, pm, seed, firstIndex, (int)(out.size() / 3), o.data()),
          "simulate");
    for (auto *g : out) g->setTransformedStatus(false);
    return 0;
  }

  // Crava::divideDataByScaleWavelet (src/crava.cpp:591-722) on the
  // real-domain stacks, closed by FFTGrid::interpolateSeismic per stack
  // (energyThreshold = ModelSettings::getEnergyThreshold).  relThick:
  // [nyp][nxp] Simbox::getRelThick; shift / gain: [ntheta][ny][nx] or null.
  int divideDataByScaleWavelet(FFTGridDevice **data, FFTGridDevice *covAlpha, const double *relThick,
                               int nx, int ny, float dz, float energyThreshold,
                               const float *shift = nullptr, const float *gain = nullptr) {
    std::vector<float *> d(nt_);
    for (int l = 0; l < nt_; ++l) d[l] = data[l]->devicePtr();
    check(crava_gpu_divide_data_by_scale_wavelet(ctx_, d.data(), covAlpha->devicePtr(), relThick, nx, ny, dz,
                                                 shift, gain),
          "divideDataByScaleWavelet");
    for (int l = 0; l < nt_; ++l)
      check(crava_gpu_interpolate_seismic(ctx_, d[l], nx, ny, energyThreshold, nullptr, nullptr),
            "interpolateSeismic");
    return 0;
  }

  // Crava::multiplyDataByScaleWaveletAndWriteToFile (src/crava.cpp:819-885)
  // up to the write: the residual spectra back in the time domain, each
  // simbox trace times its local wavelet's conjugate spectrum.
  int multiplyDataByScaleWavelet(FFTGridDevice **resid, const double *relThick, int nx, int ny, float dz,
                                 const float *shift = nullptr, const float *gain = nullptr) {
    std::vector<float *> d(nt_);
    for (int l = 0; l < nt_; ++l) d[l] = resid[l]->devicePtr();
    check(crava_gpu_multiply_data_by_scale_wavelet(ctx_, d.data(), relThick, nx, ny, dz, shift, gain),
          "multiplyDataByScaleWavelet");
    for (int l = 0; l < nt_; ++l) resid[l]->setTransformedStatus(false);
    return 0;
  }

  crava_gpu_stats stats() {
    crava_gpu_stats s{};
    check(crava_gpu_get_stats(ctx_, &s), "get_stats");
    return s;
  }

 private:
  crava_gpu_ctx *ctx_ = nullptr;
  cudaStream_t stream_ = nullptr;
  int nt_ = 0;
};

// State4D (src/state4d.h:44-106) on device grids: static and dynamic means
// and the static-static, dynamic-dynamic and static-dynamic covariance
// blocks, all holding Fourier-domain spectra, in the reference's orders.
// The current state's covariance grids are passed in the crava_gpu_grids
// order (covAlpha, covBeta, covRho, crCovAlphaBeta, crCovAlphaRho,
// crCovBetaRho).
class State4DDevice {
 public:
  FFTGridDevice *mu_static[3] = {}, *mu_dynamic[3] = {};
  FFTGridDevice *cov_ss[6] = {}, *cov_dd[6] = {}, *cov_sd[9] = {};

  // State4D::merge (src/state4d.cpp:90-159); mu == nullptr: mergeCov.
  void merge(CravaDevice &c, FFTGridDevice *mu[3], FFTGridDevice *cov[6]) {
    crava_gpu_state4d st = raw();
    float *m[3], *v[6];
    for (int i = 0; i < 3; ++i) m[i] = mu ? mu[i]->devicePtr() : nullptr;
    for (int i = 0; i < 6; ++i) v[i] = cov[i]->devicePtr();
    check(crava_gpu_state4d_merge(c.ctx(), &st, mu ? m : nullptr, v), "State4D::merge");
    for (int i = 0; i < 6; ++i) cov[i]->setTransformedStatus(true);
    if (mu)
      for (int i = 0; i < 3; ++i) mu[i]->setTransformedStatus(true);
  }

  // State4D::split (src/state4d.cpp:251-525); returns the shortcut bins.
  long long split(CravaDevice &c, FFTGridDevice *mu[3], FFTGridDevice *cov[6]) {
    crava_gpu_state4d st = raw();
    const float *m[3], *v[6];
    for (int i = 0; i < 3; ++i) m[i] = mu[i]->devicePtr();
    for (int i = 0; i < 6; ++i) v[i] = cov[i]->devicePtr();
    long long n = 0;
    check(crava_gpu_state4d_split(c.ctx(), &st, m, v, &n), "State4D::split");
    return n;
  }

  // State4D::evolve (src/state4d.cpp:527-730); lambda: the transformed
  // correlation of the time increment.
  void evolve(CravaDevice &c, const double E[36], const double meanCorr[6], const double covCorr[36],
              FFTGridDevice &lambda) {
    crava_gpu_state4d st = raw();
    check(crava_gpu_state4d_evolve(c.ctx(), &st, E, meanCorr, covCorr, lambda.devicePtr()),
          "State4D::evolve");
  }

  // ModelGeneral::advanceTime (src/modelgeneral.cpp:4722-4736); on return
  // mu and cov hold the next prior in the time domain.
  long long advanceTime(CravaDevice &c, int timeStep, int nx, int ny, const double E[36],
                        const double meanCorr[6], const double covCorr[36], FFTGridDevice *mu[3],
                        FFTGridDevice *cov[6], FFTGridDevice &work) {
    crava_gpu_state4d st = raw();
    float *m[3], *v[6];
    for (int i = 0; i < 3; ++i) m[i] = mu[i]->devicePtr();
    for (int i = 0; i < 6; ++i) v[i] = cov[i]->devicePtr();
    long long n = 0;
    check(crava_gpu_state4d_advance_time(c.ctx(), &st, timeStep, nx, ny, E, meanCorr, covCorr, m, v,
                                         work.devicePtr(), &n),
          "ModelGeneral::advanceTime");
    for (int i = 0; i < 3; ++i) mu[i]->setTransformedStatus(false);
    for (int i = 0; i < 6; ++i) cov[i]->setTransformedStatus(false);
    return n;
  }

 private:
  crava_gpu_state4d raw() const {
    crava_gpu_state4d st{};
    for (int i = 0; i < 3; ++i) {
      st.mu_static[i] = mu_static[i]->devicePtr();
      st.mu_dynamic[i] = mu_dynamic[i]->devicePtr();
    }
    for (int i = 0; i < 6; ++i) {
      st.cov_ss[i] = cov_ss[i]->devicePtr();
      st.cov_dd[i] = cov_dd[i]->devicePtr();
    }
    for (int i = 0; i < 9; ++i) st.cov_sd[i] = cov_sd[i]->devicePtr();
    return st;
  }
};

}  // namespace crava_b200
