// Test infrastructure only: a C-ABI shim around the UNMODIFIED reference
// headers (WassersteinDictionaryLearning, cpp/*.h), compiled from their
// original location by oracle/Makefile into oracle/_ref/.  Nothing in the
// product links this file; tests, smoke() and bench.py's CPU arms use it as
// the checker and the timed CPU baseline.
//
// Compiled twice: once as the kernel-domain build (Gaussian2DKernel,
// GaussianSSE2DKernel, Gaussian3DKernel) and once with
// -DCOMPUTE_BARYCENTER_LOG (LogSignArrayGaussian2DKernel), because
// evaluate_both picks the log path with that macro
// (cpp/inverseWasserstein.h:1063-1068).
#include <cstdio>
#include <cstring>
#include <unistd.h>
#include <fcntl.h>
#include <vector>
#include "inverseWasserstein.h"

namespace {

// The reference prints per-histogram progress to stdout
// (cpp/inverseWasserstein.h:1055, :1121-1122); silence fd 1 around calls.
struct Mute {
  int saved = -1;
  explicit Mute(bool on) {
    if (!on) return;
    fflush(stdout);
    std::cout.flush();
    saved = dup(1);
    int nul = open("/dev/null", O_WRONLY);
    dup2(nul, 1);
    close(nul);
  }
  ~Mute() {
    if (saved < 0) return;
    fflush(stdout);
    std::cout.flush();
    dup2(saved, 1);
    close(saved);
  }
};

template <class Kern>
BaseLoss<Kern>* make_loss(int loss_type, Kern& k) {
  switch (loss_type) {
    case 1: return new TVLoss<Kern>(k);
    case 2: return new QuadraticLoss<Kern>(k);
    case 3: return new WassersteinLoss<Kern>(k);
    case 4: return new KLLoss<Kern>(k);
    default: return nullptr;
  }
}

// Builds Problem + WassersteinRegression exactly like main_dictionary_learning.cpp:183-203.
template <class Kern>
struct Session {
  std::vector<std::vector<double>> bases;
  std::vector<double> observed;
  Problem<Kern>* problem = nullptr;
  BaseLoss<Kern>* loss = nullptr;
  ExportHistogramToCSV exporter{"/tmp"};
  WassersteinRegression<Kern>* reg = nullptr;

  Session(const Kern& kern, int P, int K, int L, int loss_type, double scale_dic,
          const double* atoms, const double* weights0, const double* obs, bool warm) {
    const size_t N = kern.N;
    bases.assign(K, std::vector<double>(N));
    for (int k = 0; k < K; ++k)
      for (size_t j = 0; j < N; ++j) bases[k][j] = atoms ? atoms[k * N + j] : 1.0 / N;
    observed.assign(obs, obs + (size_t)P * N);
    problem = new Problem<Kern>(bases, observed, kern, const_cast<double*>(weights0), P);
    loss = make_loss<Kern>(loss_type, problem->kernel);
    reg = new WassersteinRegression<Kern>(problem, L, GRADIENT_SINKHORN, *loss, exporter,
                                          scale_dic, false, false, true, warm);
    reg->exportEveryMIter = 1;
    reg->exp_weight = true;
    reg->wrTotalIteration = 1;
    if (warm) {
      reg->b_storage.assign((size_t)K * N * P, 1.0);
      reg->b_temp.assign((size_t)K * N * P, 0.0);
      reg->b.resize((size_t)K * N * (L + 1));
      std::fill(reg->b.begin(), reg->b.begin() + (size_t)K * N, 1.0);
    }
  }
  ~Session() {
    delete reg;
    delete loss;
    delete problem;
  }
};

}  // namespace

#define REF_API extern "C"

#ifndef COMPUTE_BARYCENTER_LOG
typedef Gaussian2DKernel K2;
typedef GaussianSSE2DKernel K2S;
typedef Gaussian3DKernel K3;

// Gaussian2DKernel::convolve (cpp/kernels.h:669-699) or the AVX variant (:878-897).
REF_API int ref_convolve2d(int sse, double gamma, int W, int H, const double* u, double* out, int nv) {
  if (sse) {
    // dotp_full uses aligned AVX loads (cpp/sse_helpers.h:223): it needs W and H
    // multiples of 4 and 32-byte aligned rows.
    if (W % 4 || H % 4) return -1;
    const size_t n = (size_t)W * H * nv;
    double* ua = (double*)aligned_alloc(64, ((n * sizeof(double) + 63) / 64) * 64);
    double* oa = (double*)aligned_alloc(64, ((n * sizeof(double) + 63) / 64) * 64);
    memcpy(ua, u, n * sizeof(double));
    K2S k(gamma, W, H);
    k.convolve(ua, oa, nv);
    memcpy(out, oa, n * sizeof(double));
    free(ua);
    free(oa);
  } else {
    K2 k(gamma, W, H);
    k.convolve(u, out, nv);
  }
  return 0;
}

// Gaussian3DKernel::convolve (cpp/kernels.h:762-807).
REF_API int ref_convolve3d(double gamma, int W, int H, int D, const double* u, double* out, int nv) {
  K3 k(gamma, W, H, D);
  k.convolve(u, out, nv);
  return 0;
}

template <class Kern>
static int grad_both(const Kern& kern, int K, int L, int loss_type, const double* atoms,
                     const double* lambdas, const double* obs, double* resultLa, double* resultDic,
                     double* bary) {
  Session<Kern> s(kern, 1, K, L, loss_type, 1.0, atoms, lambdas, obs, false);
  s.reg->compute_gradient_both(resultLa, resultDic, bary, 0);
  return 0;
}

// One histogram through compute_gradient_both (cpp/inverseWasserstein.h:544-674):
// raw resultLa[K], resultDic[K*N] (before the simplex projections of
// evaluate_both) and the barycenter[N].
REF_API int ref_gradient_both(int kind, double gamma, int W, int H, int D, int K, int L, int loss_type,
                      const double* atoms, const double* lambdas, const double* obs,
                      double* resultLa, double* resultDic, double* bary) {
  if (kind == 0) return grad_both(K2(gamma, W, H), K, L, loss_type, atoms, lambdas, obs, resultLa, resultDic, bary);
  if (kind == 1) return grad_both(K2S(gamma, W, H), K, L, loss_type, atoms, lambdas, obs, resultLa, resultDic, bary);
  if (kind == 2) return grad_both(K3(gamma, W, H, D), K, L, loss_type, atoms, lambdas, obs, resultLa, resultDic, bary);
  return -1;
}

template <class Kern>
static int bary_fwd(const Kern& kern, int K, int L, const double* atoms, const double* lambdas,
                    double* bary) {
  std::vector<std::vector<double>> bases(K, std::vector<double>(kern.N));
  for (int k = 0; k < K; ++k)
    for (size_t j = 0; j < kern.N; ++j) bases[k][j] = atoms[k * kern.N + j];
  std::vector<double> obs(kern.N, 0.0);
  Problem<Kern> prob(bases, obs, kern, const_cast<double*>(lambdas), 1);
  WassersteinBarycenter<Kern> wb(&prob, L);
  wb.compute_barycenter(0);
  memcpy(bary, wb.get_barycenter().data(), kern.N * sizeof(double));
  return 0;
}

// WassersteinBarycenter::compute_barycenter (cpp/inverseWasserstein.h:115-153).
REF_API int ref_barycenter(int kind, double gamma, int W, int H, int D, int K, int L, const double* atoms,
                   const double* lambdas, double* bary) {
  if (kind == 0) return bary_fwd(K2(gamma, W, H), K, L, atoms, lambdas, bary);
  if (kind == 1) return bary_fwd(K2S(gamma, W, H), K, L, atoms, lambdas, bary);
  if (kind == 2) return bary_fwd(K3(gamma, W, H, D), K, L, atoms, lambdas, bary);
  return -1;
}

template <class Kern>
static double eval_both(const Kern& kern, int P, int K, int L, int loss_type, double scale_dic,
                        const double* x, double* g, const double* obs, int quiet) {
  const size_t N = kern.N;
  Session<Kern> s(kern, P, K, L, loss_type, scale_dic, x + (size_t)P * K, x, obs, false);
  Mute m(quiet != 0);
  return WassersteinRegression<Kern>::evaluate_both(s.reg, x, g, P * K + K * (int)N, 0.0);
}

// evaluate_both (cpp/inverseWasserstein.h:986-1145) on x = [P*K log-weights*scale, K*N log-atoms].
REF_API double ref_evaluate_both(int kind, double gamma, int W, int H, int D, int P, int K, int L,
                         int loss_type, double scale_dic, const double* x, double* g,
                         const double* obs, int quiet) {
  if (kind == 0) return eval_both(K2(gamma, W, H), P, K, L, loss_type, scale_dic, x, g, obs, quiet);
  if (kind == 1) return eval_both(K2S(gamma, W, H), P, K, L, loss_type, scale_dic, x, g, obs, quiet);
  if (kind == 2) return eval_both(K3(gamma, W, H, D), P, K, L, loss_type, scale_dic, x, g, obs, quiet);
  return 0.0 / 0.0;
}

// Warm-restart evaluate_both: b_storage[P*K*N] in, b_temp[P*K*N] out
// (cpp/inverseWasserstein.h:1057-1061, :1081-1085).
REF_API double ref_evaluate_both_warm(int kind, double gamma, int W, int H, int P, int K, int L,
                              int loss_type, double scale_dic, const double* x, double* g,
                              const double* obs, const double* b_storage, double* b_last,
                              int quiet) {
  if (kind != 0) return 0.0 / 0.0;
  K2 kern(gamma, W, H);
  const size_t N = kern.N;
  Session<K2> s(kern, P, K, L, loss_type, scale_dic, x + (size_t)P * K, x, obs, true);
  std::copy(b_storage, b_storage + (size_t)P * K * N, s.reg->b_storage.begin());
  Mute m(quiet != 0);
  double f = WassersteinRegression<K2>::evaluate_both(s.reg, x, g, P * K + K * (int)N, 0.0);
  std::copy(s.reg->b_temp.begin(), s.reg->b_temp.end(), b_last);
  return f;
}

// Full regress_both (cpp/inverseWasserstein.h:362-521) with liblbfgs; `solution`
// holds [weights, atoms] in the original domain on entry and on exit.
REF_API int ref_regress_both(double gamma, int W, int H, int P, int K, int L, int loss_type,
                     double scale_dic, int max_iter, double* solution, const double* obs,
                     int quiet) {
  K2 kern(gamma, W, H);
  Session<K2> s(kern, P, K, L, loss_type, scale_dic, solution + (size_t)P * K, solution, obs, false);
  s.reg->wrTotalIteration = max_iter;
  Mute m(quiet != 0);
  s.reg->regress_both(solution);
  return 0;
}

// Loss values and gradients of cpp/loss.h.
REF_API double ref_loss(int loss_type, double gamma, int W, int H, const double* v1, const double* v2,
                double* grad) {
  K2 kern(gamma, W, H);
  BaseLoss<K2>* l = make_loss<K2>(loss_type, kern);
  if (!l) return 0.0 / 0.0;
  double r = l->loss(v1, v2, (int)kern.N);
  l->gradient(v1, v2, (int)kern.N, grad);
  delete l;
  return r;
}

REF_API int ref_is_log_build(void) { return 0; }

#else  // COMPUTE_BARYCENTER_LOG
typedef LogSignArrayGaussian2DKernel KL2;

// log_convolve (cpp/kernels.h:1073-1112).
REF_API int ref_log_convolve2d(double gamma, int W, int H, const double* u, double* out, int nv) {
  KL2 k(gamma, W, H);
  k.log_convolve(u, out, nv);
  return 0;
}

// log_convolve_signArray (cpp/kernels.h:1117-1159); signs are read and overwritten.
REF_API int ref_log_convolve2d_signed(double gamma, int W, int H, const double* u, unsigned char* signs,
                              double* out, int nv) {
  KL2 k(gamma, W, H);
  k.log_convolve_signArray(u, signs, out, nv);
  return 0;
}

// compute_gradient_both_log_signArray (cpp/inverseWasserstein.h:678-814).
REF_API int ref_gradient_both_log(double gamma, int W, int H, int K, int L, int loss_type,
                          const double* atoms, const double* lambdas, const double* obs,
                          double* resultLa, double* resultDic, double* bary) {
  KL2 kern(gamma, W, H);
  Session<KL2> s(kern, 1, K, L, loss_type, 1.0, atoms, lambdas, obs, false);
  s.reg->compute_gradient_both_log_signArray(resultLa, resultDic, bary, 0);
  return 0;
}

// compute_barycenter_log (cpp/inverseWasserstein.h:155-201).
REF_API int ref_barycenter_log(double gamma, int W, int H, int K, int L, const double* atoms,
                       const double* lambdas, double* bary) {
  KL2 kern(gamma, W, H);
  std::vector<std::vector<double>> bases(K, std::vector<double>(kern.N));
  for (int k = 0; k < K; ++k)
    for (size_t j = 0; j < kern.N; ++j) bases[k][j] = atoms[k * kern.N + j];
  std::vector<double> obs(kern.N, 0.0);
  Problem<KL2> prob(bases, obs, kern, const_cast<double*>(lambdas), 1);
  WassersteinBarycenter<KL2> wb(&prob, L);
  wb.compute_barycenter_log(0);
  memcpy(bary, wb.get_barycenter().data(), kern.N * sizeof(double));
  return 0;
}

// evaluate_both through the log-domain path (-DCOMPUTE_BARYCENTER_LOG).
REF_API double ref_evaluate_both_log(double gamma, int W, int H, int P, int K, int L, int loss_type,
                             double scale_dic, const double* x, double* g, const double* obs,
                             int quiet) {
  KL2 kern(gamma, W, H);
  const size_t N = kern.N;
  Session<KL2> s(kern, P, K, L, loss_type, scale_dic, x + (size_t)P * K, x, obs, false);
  Mute m(quiet != 0);
  return WassersteinRegression<KL2>::evaluate_both(s.reg, x, g, P * K + K * (int)N, 0.0);
}

REF_API int ref_is_log_build(void) { return 1; }
#endif

REF_API int ref_omp_threads(void) {
#ifdef HAS_OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

