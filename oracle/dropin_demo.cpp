// Test infrastructure: the reference's own C++ classes instantiated on the CUDA
// KernelType of include/wdl_kernels.hpp, next to the reference's CPU kernel.
// Built by oracle/Makefile against the unmodified reference headers into
// oracle/_ref/dropin_demo (linked to the product library libwdl_b200.so);
// tests/test_gpu_dropin.py runs it on a GPU and checks its exit status.
//
// Checks, on seeded inputs (P=3 histograms of 24x20, K=3, L=8, quadratic loss):
//  1. compute_gradient_both of WassersteinRegression<CudaGaussian2DKernel>
//     (the reference template, every convolve a device call) vs
//     WassersteinRegression<Gaussian2DKernel>;
//  2. the specialised device-resident evaluate_both vs the reference's;
//  3. three L-BFGS iterations of the reference's regress_both on each.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "inverseWasserstein.h"
#define WDL_SPECIALIZE_REGRESSION
#include "wdl_kernels.hpp"

namespace {

double rel(const std::vector<double>& a, const std::vector<double>& b) {
  double num = 0, den = 1e-300;
  for (size_t i = 0; i < a.size(); ++i) {
    num = std::max(num, std::fabs(a[i] - b[i]));
    den = std::max(den, std::fabs(b[i]));
  }
  return num / den;
}

struct Lcg {
  unsigned long long s;
  double next() {
    s = s * 6364136223846793005ULL + 1442695040888963407ULL;
    return ((s >> 11) & ((1ULL << 53) - 1)) / 9007199254740992.0;
  }
};

template <class Kern>
struct Setup {
  std::vector<std::vector<double>> bases;
  std::vector<double> obs, w;
  Problem<Kern>* prob;
  QuadraticLoss<Kern> loss;
  ExportHistogramToCSV exporter{"/tmp"};
  WassersteinRegression<Kern>* reg;
  Setup(const Kern& k, int P, int K, int L, const std::vector<double>& atoms,
        const std::vector<double>& weights, const std::vector<double>& observed, double sd) {
    const size_t N = k.N;
    bases.assign(K, std::vector<double>(N));
    for (int i = 0; i < K; ++i)
      for (size_t j = 0; j < N; ++j) bases[i][j] = atoms[i * N + j];
    obs = observed;
    w = weights;
    prob = new Problem<Kern>(bases, obs, k, w.data(), P);
    reg = new WassersteinRegression<Kern>(prob, L, GRADIENT_SINKHORN, loss, exporter, sd, false,
                                          false, true, false);
    reg->exp_weight = true;
    reg->wrTotalIteration = 3;
  }
  ~Setup() {
    delete reg;
    delete prob;
  }
};

}  // namespace

int main() {
  const int W = 24, H = 20, P = 3, K = 3, L = 8;
  const size_t N = (size_t)W * H;
  const double gamma = 2.0, sd = (N / (double)P) / 100.0;
  Lcg rng{42};
  std::vector<double> atoms(K * N), weights(P * K), obs(P * N);
  for (auto& a : atoms) a = 1.0 + 0.1 * rng.next();
  for (auto& v : weights) v = rng.next();
  for (int p = 0; p < P; ++p) {  // one smooth bump per histogram plus a floor
    const double cx = W * (0.3 + 0.4 * rng.next()), cy = H * (0.3 + 0.4 * rng.next());
    double s = 0;
    for (int y = 0; y < H; ++y)
      for (int x = 0; x < W; ++x) {
        const double v = std::exp(-((x - cx) * (x - cx) + (y - cy) * (y - cy)) / 18.0) + 1e-6;
        obs[p * N + y * W + x] = v;
        s += v;
      }
    for (size_t j = 0; j < N; ++j) obs[p * N + j] /= s;
  }
  int fails = 0;

  // 1. The reference template on the CUDA KernelType (per-convolve device calls).
  {
    Gaussian2DKernel kc(gamma, W, H);
    CudaGaussian2DKernel kg(gamma, W, H, WDL_FP64);
    Setup<Gaussian2DKernel> a(kc, 1, K, L, atoms, weights, obs, sd);
    Setup<CudaGaussian2DKernel> b(kg, 1, K, L, atoms, weights, obs, sd);
    std::vector<double> la_a(K), la_b(K), dic_a(K * N), dic_b(K * N), by_a(N), by_b(N);
    a.reg->compute_gradient_both(la_a.data(), dic_a.data(), by_a.data(), 0);
    b.reg->compute_gradient_both(la_b.data(), dic_b.data(), by_b.data(), 0);
    const double e1 = rel(by_b, by_a), e2 = rel(dic_b, dic_a), e3 = rel(la_b, la_a);
    std::printf("kerneltype compute_gradient_both: bary %.2e dic %.2e la %.2e\n", e1, e2, e3);
    if (!(e1 < 1e-10 && e2 < 1e-10 && e3 < 1e-8)) ++fails;
  }
  // 2./3. Device-resident evaluate_both and regress_both.
  {
    Gaussian2DKernel kc(gamma, W, H);
    CudaGaussian2DKernel kg(gamma, W, H, WDL_FP64);
    Setup<Gaussian2DKernel> a(kc, P, K, L, atoms, weights, obs, sd);
    Setup<CudaGaussian2DKernel> b(kg, P, K, L, atoms, weights, obs, sd);
    const int n = P * K + K * (int)N;
    std::vector<double> x(n), ga(n), gb(n);
    for (int i = 0; i < P * K; ++i) x[i] = std::log(weights[i]) * sd;
    for (size_t i = 0; i < K * N; ++i) x[P * K + i] = std::log(atoms[i]);
    FILE* keep = stdout;
    stdout = std::fopen("/dev/null", "w");  // the reference prints progress
    const double fa = WassersteinRegression<Gaussian2DKernel>::evaluate_both(a.reg, x.data(), ga.data(), n, 0);
    const double fb = WassersteinRegression<CudaGaussian2DKernel>::evaluate_both(b.reg, x.data(), gb.data(), n, 0);
    std::vector<double> sa(n), sb(n);
    for (int i = 0; i < P * K; ++i) sa[i] = sb[i] = weights[i] / (weights[(i / K) * K] + weights[(i / K) * K + 1] + weights[(i / K) * K + 2]);
    for (size_t i = 0; i < K * N; ++i) sa[P * K + i] = sb[P * K + i] = atoms[i];
    std::cout.setstate(std::ios::failbit);
    a.reg->regress_both(sa.data());
    b.reg->regress_both(sb.data());
    std::cout.clear();
    std::fclose(stdout);
    stdout = keep;
    std::vector<double> gaa(ga.begin() + P * K, ga.end()), gba(gb.begin() + P * K, gb.end());
    const double ef = std::fabs(fb - fa) / std::fabs(fa), eg = rel(gba, gaa), es = rel(sb, sa);
    std::printf("evaluate_both: f %.2e atom-grad %.2e; regress_both (3 it): solution %.2e\n", ef,
                eg, es);
    if (!(ef < 1e-10 && eg < 1e-10 && es < 1e-8)) ++fails;
  }
  std::printf(fails ? "FAIL\n" : "OK\n");
  return fails ? 1 : 0;
}
