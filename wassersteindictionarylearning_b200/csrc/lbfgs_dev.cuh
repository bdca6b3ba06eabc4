// The device restatement of liblbfgs (cpp/lbfgs/lbfgs.c:256-654, with the
// strong-Wolfe backtracking line search of :772-867) that the batched weight
// fits run: one state machine per optimisation, advanced once per objective
// evaluation, making liblbfgs' decisions in liblbfgs' order.  Shared by the
// round-based fit (fit.cu) and the persistent log-domain fit (fit_log.cu).
//
// Variables: x in R^K, weights = softmax(x) (the reference's exp_weight
// transform with scaleDictionary 1 followed by the normalisation by the sum,
// cpp/inverseWasserstein.h:1000-1020); gradient = (la - <w, la>) * w, the
// projection and chain rule of evaluate_both (:1092-1097, :1124-1133).
#pragma once

#include "wdl_internal.cuh"

namespace wdl {
namespace lbdev {

constexpr int kM = 6;  // correction pairs (liblbfgs default, kept by the reference)

// liblbfgs return codes (cpp/lbfgs/lbfgs.h:74-147)
constexpr int kSuccess = 0, kAlreadyMinimized = 2, kMinimumStep = -1000, kMaximumStep = -999,
              kMaximumLinesearch = -998, kMaximumIteration = -997, kInvalidParameters = -995,
              kIncreaseGradient = -994;

struct LbParam {
  int max_iterations, max_linesearch;
  double epsilon, ftol, wolfe, min_step, max_step;
};

struct LbState {
  int K, phase;  // phase: 0 first evaluation pending, 1 line-search trial pending, 2 done
  int k, end, count, status, evals;
  double f, finit, dginit, step, fret;
};

// Doubles of state per optimisation: x, g, xp, gp, d [K each], s[m][K],
// y[m][K], ys[m], alpha[m].
__host__ __device__ inline size_t pool_doubles(int K) { return (size_t)(5 + 2 * kM) * K + 2 * kM; }

__device__ inline double dotk(const double* a, const double* b, int K) {
  double s = 0;
  for (int k = 0; k < K; ++k) s += a[k] * b[k];
  return s;
}

// weights = softmax(x) into w64 (and w32 when given)
__device__ inline void softmax_weights(const double* x, int K, double* w64, float* w32) {
  double mx = x[0];
  for (int k = 1; k < K; ++k) mx = x[k] > mx ? x[k] : mx;
  double s = 0;
  for (int k = 0; k < K; ++k) s += exp(x[k] - mx);
  for (int k = 0; k < K; ++k) {
    const double w = exp(x[k] - mx) / s;
    w64[k] = w;
    if (w32) w32[k] = (float)w;
  }
}

// Consume the evaluation (f, la = raw weight gradient resultLa) at the
// current trial point, whose weights are w64; move to the next trial point
// (written to w64 / w32) or finish (o.phase == 2).  A non-finite evaluation
// finishes with status `nonfinite_status`.
__device__ inline void lbfgs_advance(LbState& o, double* v, double f, const double* la, double* w64,
                                     float* w32, const LbParam& prm, int nonfinite_status) {
  const int K = o.K;
  double* x = v;
  double* g = x + K;
  double* xp = x + 2 * K;
  double* gp = x + 3 * K;
  double* d = x + 4 * K;
  double* S = x + 5 * K;
  double* Y = S + kM * K;
  double* ys_h = Y + kM * K;
  double* alpha = ys_h + kM;

  o.evals++;
  bool finite = isfinite(f);
  double wla = 0;
  for (int k = 0; k < K; ++k) {
    finite = finite && isfinite(la[k]);
    wla += w64[k] * la[k];
  }
  auto finish = [&](int status, double fret) {
    o.status = status;
    o.fret = fret;
    o.phase = 2;
  };
  if (!finite) {
    finish(nonfinite_status, f);
    return;
  }
  for (int k = 0; k < K; ++k) g[k] = (la[k] - wla) * w64[k];

  // start of a line search from the accepted point x (lbfgs.c:772-790)
  auto start_ls = [&]() {
    for (int k = 0; k < K; ++k) {
      xp[k] = x[k];
      gp[k] = g[k];
    }
    o.finit = o.f;
    if (o.step <= 0) {
      finish(kInvalidParameters, o.f);
      return;
    }
    o.dginit = dotk(g, d, K);
    if (o.dginit > 0) {
      finish(kIncreaseGradient, o.f);
      return;
    }
    o.count = 0;
    for (int k = 0; k < K; ++k) x[k] = xp[k] + o.step * d[k];
    softmax_weights(x, K, w64, w32);
    o.phase = 1;
  };

  if (o.phase == 0) {  // first evaluation (lbfgs.c:423-470)
    o.f = f;
    const double xnorm = fmax(sqrt(dotk(x, x, K)), 1.0);
    const double gnorm = sqrt(dotk(g, g, K));
    if (gnorm / xnorm <= prm.epsilon) {
      finish(kAlreadyMinimized, f);
    } else {
      for (int k = 0; k < K; ++k) d[k] = -g[k];
      o.step = 1.0 / sqrt(dotk(d, d, K));
      o.k = 1;
      o.end = 0;
      start_ls();
    }
    return;
  }
  // a line-search trial (lbfgs.c:791-867)
  o.count++;
  double width = 0;
  bool accept = false;
  if (f > o.finit + o.step * prm.ftol * o.dginit) {
    width = 0.5;
  } else {
    const double dg = dotk(g, d, K);
    if (dg < prm.wolfe * o.dginit) width = 2.1;
    else if (dg > -prm.wolfe * o.dginit) width = 0.5;
    else accept = true;
  }
  if (!accept) {
    int fail = 0;
    if (o.step < prm.min_step) fail = kMinimumStep;
    else if (o.step > prm.max_step) fail = kMaximumStep;
    else if (prm.max_linesearch <= o.count) fail = kMaximumLinesearch;
    if (fail) {  // revert to the previous point (lbfgs.c:487-492)
      for (int k = 0; k < K; ++k) x[k] = xp[k];
      finish(fail, o.finit);
    } else {
      o.step *= width;
      for (int k = 0; k < K; ++k) x[k] = xp[k] + o.step * d[k];
      softmax_weights(x, K, w64, w32);
    }
    return;
  }
  // accepted: convergence tests, then the next direction (lbfgs.c:505-612)
  o.f = f;
  const double xnorm = sqrt(dotk(x, x, K));
  const double gnorm = sqrt(dotk(g, g, K));
  if (gnorm / fmax(xnorm, 1.0) <= prm.epsilon) {
    finish(kSuccess, f);
    return;
  }
  if (prm.max_iterations != 0 && prm.max_iterations < o.k + 1) {
    finish(kMaximumIteration, f);
    return;
  }
  double* s_e = S + (size_t)o.end * K;
  double* y_e = Y + (size_t)o.end * K;
  for (int k = 0; k < K; ++k) {
    s_e[k] = x[k] - xp[k];
    y_e[k] = g[k] - gp[k];
  }
  const double ys = dotk(y_e, s_e, K);
  const double yy = dotk(y_e, y_e, K);
  ys_h[o.end] = ys;
  const int bound = o.k < kM ? o.k : kM;
  o.k++;
  o.end = (o.end + 1) % kM;
  for (int k = 0; k < K; ++k) d[k] = -g[k];
  int j = o.end;
  for (int b = 0; b < bound; ++b) {
    j = (j + kM - 1) % kM;
    alpha[j] = dotk(S + (size_t)j * K, d, K) / ys_h[j];
    for (int k = 0; k < K; ++k) d[k] -= alpha[j] * Y[(size_t)j * K + k];
  }
  for (int k = 0; k < K; ++k) d[k] *= ys / yy;
  for (int b = 0; b < bound; ++b) {
    const double beta = dotk(Y + (size_t)j * K, d, K) / ys_h[j];
    for (int k = 0; k < K; ++k) d[k] += (alpha[j] - beta) * S[(size_t)j * K + k];
    j = (j + 1) % kM;
  }
  o.step = 1.0;
  start_ls();
}

}  // namespace lbdev
}  // namespace wdl
