// wdl_kernels.hpp — C++ host drop-in over the C ABI of wdl.h.
//
// 1. KernelType classes with the reference's duck-typed interface
//    (cpp/kernels.h: N, gamma, W_, H_, convolve, convolveAdjoint, operator(),
//    and the log-domain members), so that Problem / WassersteinBarycenter /
//    WassersteinRegression / the loss functors instantiate on them unchanged:
//      CudaGaussian2DKernel              for Gaussian2DKernel / GaussianSSE2DKernel
//      CudaGaussian3DKernel              for Gaussian3DKernel
//      CudaLogSignArrayGaussian2DKernel  for LogSignArrayGaussian2DKernel
//    Copies share one device context (the reference's Problem copies its kernel,
//    cpp/inverseWasserstein.h:37).  Each convolve call is one host<->device
//    round trip: correct everywhere, but the device-resident path below is the
//    one to use for throughput.
//
// 2. With WDL_SPECIALIZE_REGRESSION defined and the reference's
//    inverseWasserstein.h included first, an explicit specialisation of
//    WassersteinRegression<CudaGaussian2DKernel>::evaluate_both replaces the
//    serial per-histogram loop (cpp/inverseWasserstein.h:1052-1113) with one
//    wdl_evaluate_both call for all P histograms; liblbfgs, regress_both,
//    progress_both and the exporters stay the reference's own.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "wdl.h"

namespace wdl_host {

struct Context {
  wdl_ctx* ctx = nullptr;
  ~Context() {
    if (ctx) wdl_destroy(ctx);
  }
};

inline std::shared_ptr<Context> make_context(int W, int H, int D, double gamma, int precision,
                                             int domain) {
  auto c = std::make_shared<Context>();
  if (W <= 0 || H <= 0) return c;  // default-constructed kernel: no device context yet
  const int rc = wdl_create(&c->ctx, -1, W, H, D, gamma, precision, domain);
  if (rc != WDL_OK)
    throw std::runtime_error(std::string("wdl_create: ") + wdl_strerror(rc) + ": " +
                             wdl_last_error(nullptr));
  return c;
}

inline void check(int rc, const wdl_ctx* ctx, const char* what) {
  if (rc != WDL_OK)
    throw std::runtime_error(std::string(what) + ": " + wdl_strerror(rc) + ": " + wdl_last_error(ctx));
}

inline double gibbs(double d2, double gamma) { return std::max(1e-250, std::exp(-d2 / gamma)); }

}  // namespace wdl_host

// Gaussian2DKernel drop-in (cpp/kernels.h:630-708).  precision: WDL_FP64 gives
// the reference's arithmetic (1e-10 parity); WDL_FP32 / WDL_TF32 /
// WDL_SPLIT_BF16 select the faster device forms.
class CudaGaussian2DKernel {
 public:
  CudaGaussian2DKernel(double regularization = 25., int W = 0, int H = 0, int precision = WDL_FP64)
      : gamma(regularization), W_(W), H_(H), N((size_t)W * H), precision_(precision),
        ctx_(wdl_host::make_context(W, H, 1, regularization, precision, WDL_DOMAIN_KERNEL)) {}
  double operator()(int i, int j) const {
    const int x0 = i % (int)W_, y0 = i / (int)W_, x1 = j % (int)W_, y1 = j / (int)W_;
    return wdl_host::gibbs((double)(x0 - x1) * (x0 - x1) + (double)(y0 - y1) * (y0 - y1), gamma);
  }
  void convolve(const double* u, double* result, int nvectors = 1) const {
    wdl_host::check(wdl_convolve(ctx_->ctx, u, result, nvectors), ctx_->ctx, "wdl_convolve");
  }
  void convolveAdjoint(const double* u, double* result, int nvectors = 1) const {
    convolve(u, result, nvectors);
  }
  wdl_ctx* ctx() const { return ctx_->ctx; }
  int precision() const { return precision_; }

  double gamma;
  size_t W_, H_;
  size_t N;

 private:
  int precision_;
  std::shared_ptr<wdl_host::Context> ctx_;
};

// Gaussian3DKernel drop-in (cpp/kernels.h:712-815).
class CudaGaussian3DKernel {
 public:
  CudaGaussian3DKernel(double regularization = 25., int W = 0, int H = 0, int D = 0,
                       int precision = WDL_FP64)
      : gamma(regularization), W_(W), H_(H), D_(D), N((size_t)W * H * D),
        ctx_(wdl_host::make_context(W, H, D, regularization, precision, WDL_DOMAIN_KERNEL)) {}
  double operator()(int i, int j) const {
    const int WH = (int)(W_ * H_);
    const int z0 = i / WH, z1 = j / WH;
    i -= z0 * WH;
    j -= z1 * WH;
    const int x0 = i % (int)W_, y0 = i / (int)W_, x1 = j % (int)W_, y1 = j / (int)W_;
    return wdl_host::gibbs((double)(x0 - x1) * (x0 - x1) + (double)(y0 - y1) * (y0 - y1) +
                               (double)(z0 - z1) * (z0 - z1),
                           gamma);
  }
  void convolve(const double* u, double* result, int nvectors = 1) const {
    wdl_host::check(wdl_convolve(ctx_->ctx, u, result, nvectors), ctx_->ctx, "wdl_convolve");
  }
  void convolveAdjoint(const double* u, double* result, int nvectors = 1) const {
    convolve(u, result, nvectors);
  }
  wdl_ctx* ctx() const { return ctx_->ctx; }

  double gamma;
  size_t W_, H_, D_, N;

 private:
  std::shared_ptr<wdl_host::Context> ctx_;
};

// LogSignArrayGaussian2DKernel drop-in (cpp/kernels.h:1034-1202).  The
// kernel-domain members run through a second context (the loss functors call
// convolve on any kernel type, cpp/loss.h:110-143).
class CudaLogSignArrayGaussian2DKernel {
 public:
  CudaLogSignArrayGaussian2DKernel(double regularization = 25., int W = 0, int H = 0,
                                   int precision = WDL_FP64)
      : gamma(regularization), W_(W), H_(H), N((size_t)W * H),
        ctx_(wdl_host::make_context(W, H, 1, regularization, precision, WDL_DOMAIN_LOG)),
        kctx_(wdl_host::make_context(W, H, 1, regularization, precision, WDL_DOMAIN_KERNEL)) {}
  double operator()(int i, int j) const {
    const int x0 = i % (int)W_, y0 = i / (int)W_, x1 = j % (int)W_, y1 = j / (int)W_;
    return wdl_host::gibbs((double)(x0 - x1) * (x0 - x1) + (double)(y0 - y1) * (y0 - y1), gamma);
  }
  void log_convolve(const double* log_u, double* result, int nvectors = 1) const {
    wdl_host::check(wdl_log_convolve(ctx_->ctx, log_u, result, nvectors), ctx_->ctx,
                    "wdl_log_convolve");
  }
  void log_convolveAdjoint(const double* u, double* result, int nvectors = 1) const {
    log_convolve(u, result, nvectors);
  }
  void log_convolve_signArray(const double* log_u, unsigned char* signArray, double* result,
                              int nvectors = 1) const {
    wdl_host::check(wdl_log_convolve_signed(ctx_->ctx, log_u, signArray, result, nvectors),
                    ctx_->ctx, "wdl_log_convolve_signed");
  }
  void log_convolve_signArrayAdjoint(const double* u, unsigned char* sign_array, double* result,
                                     int nvectors = 1) const {
    log_convolve_signArray(u, sign_array, result, nvectors);
  }
  void convolve(const double* u, double* result, int nvectors = 1) const {
    wdl_host::check(wdl_convolve(kctx_->ctx, u, result, nvectors), kctx_->ctx, "wdl_convolve");
  }
  void convolveAdjoint(const double* u, double* result, int nvectors = 1) const {
    convolve(u, result, nvectors);
  }
  wdl_ctx* ctx() const { return ctx_->ctx; }

  double gamma;
  size_t W_, H_;
  size_t N;

 private:
  std::shared_ptr<wdl_host::Context> ctx_, kctx_;
};

#ifdef WDL_SPECIALIZE_REGRESSION
// Device-resident evaluate_both for the CUDA kernel type: same contract as
// cpp/inverseWasserstein.h:986-1145 (x -> loss, g), one device call for all P
// histograms.  Requires the reference's inverseWasserstein.h to be included
// before this header.
namespace wdl_host {
template <class Kern>
inline int loss_index(const BaseLoss<Kern>& l) {
  if (dynamic_cast<const TVLoss<Kern>*>(&l)) return WDL_LOSS_TV;
  if (dynamic_cast<const QuadraticLoss<Kern>*>(&l)) return WDL_LOSS_QUADRATIC;
  if (dynamic_cast<const WassersteinLoss<Kern>*>(&l)) return WDL_LOSS_WASSERSTEIN;
  if (dynamic_cast<const KLLoss<Kern>*>(&l)) return WDL_LOSS_KL;
  return -1;
}
}  // namespace wdl_host

template <>
inline lbfgsfloatval_t WassersteinRegression<CudaGaussian2DKernel>::evaluate_both(
    void* instance, const lbfgsfloatval_t* variables, lbfgsfloatval_t* gradient, const int n,
    const lbfgsfloatval_t step) {
  auto* reg = static_cast<WassersteinRegression<CudaGaussian2DKernel>*>(instance);
  Problem<CudaGaussian2DKernel>* prob = reg->problem;
  const int N = (int)prob->N, K = (int)prob->K, P = prob->num_pdfs;
  const int lt = wdl_host::loss_index(reg->loss);
  if (!reg->exp_weight || lt < 0) {
    std::fprintf(stderr, "wdl: evaluate_both supports exp_weight and the four reference losses\n");
    return NAN;
  }
  const bool warm = reg->warmRestart;
  if (warm && reg->b_temp.size() < (size_t)K * N * P) reg->b_temp.resize((size_t)K * N * P);
  double f = NAN;
  const int rc = wdl_evaluate_both(prob->kernel.ctx(), P, K, reg->bary_computation->Niters, lt,
                                   reg->scaleDictionary, variables, gradient, n,
                                   prob->observed_pdf.data(), &f,
                                   warm ? reg->b_storage.data() : nullptr,
                                   warm ? reg->b_temp.data() : nullptr, nullptr);
  if (rc != WDL_OK && rc != WDL_ERR_NONFINITE) {
    std::fprintf(stderr, "wdl_evaluate_both: %s: %s\n", wdl_strerror(rc),
                 wdl_last_error(prob->kernel.ctx()));
    return NAN;  // progress_both cancels L-BFGS on NaN (:1180-1184)
  }
  // The reference leaves the normalised atoms in prob->pdfs (:1034-1038).
  for (int k = 0; k < K; ++k) {
    double s = 0;
    for (int j = 0; j < N; ++j) s += std::exp(variables[P * K + k * N + j]);
    for (int j = 0; j < N; ++j) prob->pdfs[k][j] = std::exp(variables[P * K + k * N + j]) / s;
  }
  return f;
}
#endif
