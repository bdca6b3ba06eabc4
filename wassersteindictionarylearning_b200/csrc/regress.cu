// regress_both (cpp/inverseWasserstein.h:362-423) with the L-BFGS on the device.
//
// The reference optimises x = [P*K scaled log-weights, K*N log-atoms] with
// liblbfgs (cpp/lbfgs/lbfgs.c:256-654, strong-Wolfe backtracking :772-867)
// on the host, one evaluate_both per objective evaluation.  Here the whole
// optimisation state (x, the gradient, the previous point, the direction and
// the m = 6 correction pairs, n = P*K + K*N doubles each) stays in device
// memory: a round is one evaluate_both on the device followed by one launch of
// k_regress_step, a single CTA that makes liblbfgs' decision for that
// evaluation (first evaluation, line-search trial, accepted step with the
// two-loop recursion) and writes the next trial point.  The host only reads a
// 4-byte phase word after each round to know when the run has finished; no
// vector crosses the bus.  FP64 throughout, block reductions in a fixed order
// (results are deterministic; they differ from liblbfgs' sequential sums only
// in the last bits).
//
// Warm restart (:369-423 with warmRestart): runs of 10 L-BFGS iterations, the
// scalings b[L] of each run's evaluations kept on the device and used as b[0]
// by the next run (:1057-1061, :1081-1085).
#include <cmath>

#include "wdl_internal.cuh"

namespace wdl {
namespace {

constexpr int kM = 6;           // correction pairs (liblbfgs default, kept by the reference)
constexpr int kThreads = 1024;  // the step kernel's single CTA

// liblbfgs return codes (cpp/lbfgs/lbfgs.h:74-147)
constexpr int kSuccess = 0, kAlreadyMinimized = 2, kCanceled = -1021, kMinimumStep = -1000,
              kMaximumStep = -999, kMaximumLinesearch = -998, kMaximumIteration = -997,
              kInvalidParameters = -995, kIncreaseGradient = -994;

struct RegParam {
  int max_iterations, max_linesearch;
  double epsilon, ftol, wolfe, min_step, max_step;
};

struct RegState {
  int phase;  // 0: first evaluation pending, 1: line-search trial pending, 2: done
  int k, end, count, status, evals, iterations;
  double f, finit, dginit, step;
  double ys[kM], alpha[kM];
};

struct RegVecs {
  double *x, *g, *xp, *gp, *d, *S, *Y;  // S, Y: [kM][n]
  const double* f_eval;                  // objective at x (device scalar)
  const double* g_eval;                  // gradient at x
};

// Sum over the CTA of one value per thread, in a fixed order; every thread
// gets the result.
__device__ double cta_sum(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5;
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[w] = v;
  __syncthreads();
  double t = 0;
  for (int i = 0; i < kThreads / 32; ++i) t += red[i];
  return t;
}

__device__ double dotn(const double* a, const double* b, size_t n, double* red) {
  double s = 0;
  for (size_t i = threadIdx.x; i < n; i += kThreads) s += a[i] * b[i];
  return cta_sum(s, red);
}

// Consumes the evaluation at x and moves to the next trial point or finishes.
// Control flow is uniform across the CTA (every branch depends on reduced or
// shared scalars only).
__global__ void __launch_bounds__(kThreads) k_regress_step(RegState* st, RegVecs v, size_t n, RegParam prm) {
  __shared__ double red[kThreads / 32];
  __shared__ RegState o;
  if (threadIdx.x == 0) o = *st;
  __syncthreads();
  if (o.phase == 2) return;
  double* x = v.x;
  double* g = v.g;
  double* xp = v.xp;
  double* gp = v.gp;
  double* d = v.d;
  const double f = *v.f_eval;
  for (size_t i = threadIdx.x; i < n; i += kThreads) g[i] = v.g_eval[i];
  __syncthreads();

  bool done = false;
  auto finish = [&](int status) {
    if (threadIdx.x == 0) {
      o.status = status;
      o.phase = 2;
    }
    done = true;
  };
  // x = xp + step * d
  auto move = [&]() {
    for (size_t i = threadIdx.x; i < n; i += kThreads) x[i] = xp[i] + o.step * d[i];
  };
  // revert to the line search's starting point (lbfgs.c:487-492)
  auto revert = [&]() {
    for (size_t i = threadIdx.x; i < n; i += kThreads) x[i] = xp[i];
  };
  // start a line search from the accepted point x (lbfgs.c:772-790)
  auto start_ls = [&]() {
    for (size_t i = threadIdx.x; i < n; i += kThreads) {
      xp[i] = x[i];
      gp[i] = g[i];
    }
    __syncthreads();
    if (!(o.step > 0)) {
      finish(kInvalidParameters);
      return;
    }
    const double dginit = dotn(g, d, n, red);
    if (dginit > 0) {
      finish(kIncreaseGradient);
      return;
    }
    if (threadIdx.x == 0) {
      o.finit = o.f;
      o.dginit = dginit;
      o.count = 0;
      o.phase = 1;
    }
    __syncthreads();
    move();
  };

  if (threadIdx.x == 0) o.evals++;
  if (o.phase == 0) {  // first evaluation (lbfgs.c:423-470)
    if (threadIdx.x == 0) o.f = f;
    for (size_t i = threadIdx.x; i < n; i += kThreads) d[i] = -g[i];
    __syncthreads();
    const double xnorm = fmax(sqrt(dotn(x, x, n, red)), 1.0);
    const double gnorm = sqrt(dotn(g, g, n, red));
    if (gnorm / xnorm <= prm.epsilon) {
      finish(kAlreadyMinimized);
    } else {
      const double dd = dotn(d, d, n, red);
      if (threadIdx.x == 0) {
        o.step = 1.0 / sqrt(dd);
        o.k = 1;
        o.end = 0;
      }
      __syncthreads();
      start_ls();
    }
  } else {  // a line-search trial (lbfgs.c:791-867)
    if (threadIdx.x == 0) o.count++;
    __syncthreads();
    double width = 0;
    bool accept = false;
    if (f > o.finit + o.step * prm.ftol * o.dginit) {
      width = 0.5;
    } else {
      const double dg = dotn(g, d, n, red);
      if (dg < prm.wolfe * o.dginit) width = 2.1;
      else if (dg > -prm.wolfe * o.dginit) width = 0.5;
      else accept = true;
    }
    if (!accept) {
      if (o.step < prm.min_step) {
        revert();
        finish(kMinimumStep);
      } else if (o.step > prm.max_step) {
        revert();
        finish(kMaximumStep);
      } else if (prm.max_linesearch <= o.count) {
        revert();
        finish(kMaximumLinesearch);
      } else {
        __syncthreads();
        if (threadIdx.x == 0) o.step *= width;
        __syncthreads();
        move();
      }
    } else {  // accepted step (lbfgs.c:494-612)
      if (threadIdx.x == 0) {
        o.f = f;
        o.iterations++;
      }
      const double xnorm = sqrt(dotn(x, x, n, red));
      const double gnorm = sqrt(dotn(g, g, n, red));
      if (isnan(f)) {  // progress_both cancels on a NaN loss (cpp/inverseWasserstein.h:1180-1184)
        finish(kCanceled);
      } else if (gnorm / fmax(xnorm, 1.0) <= prm.epsilon) {
        finish(kSuccess);
      } else if (prm.max_iterations != 0 && prm.max_iterations < o.k + 1) {
        finish(kMaximumIteration);
      } else {
        const int end = o.end;
        double* s_end = v.S + (size_t)end * n;
        double* y_end = v.Y + (size_t)end * n;
        for (size_t i = threadIdx.x; i < n; i += kThreads) {
          s_end[i] = x[i] - xp[i];
          y_end[i] = g[i] - gp[i];
          d[i] = -g[i];
        }
        __syncthreads();
        const double ys = dotn(y_end, s_end, n, red);
        const double yy = dotn(y_end, y_end, n, red);
        const int bound = o.k < kM ? o.k : kM;
        __syncthreads();
        if (threadIdx.x == 0) {
          o.ys[end] = ys;
          o.k++;
          o.end = (end + 1) % kM;
        }
        __syncthreads();
        int j = o.end;
        for (int it = 0; it < bound; ++it) {
          j = (j + kM - 1) % kM;
          const double a = dotn(v.S + (size_t)j * n, d, n, red) / o.ys[j];
          if (threadIdx.x == 0) o.alpha[j] = a;
          const double* yj = v.Y + (size_t)j * n;
          for (size_t i = threadIdx.x; i < n; i += kThreads) d[i] -= a * yj[i];
          __syncthreads();
        }
        const double scale = ys / yy;
        for (size_t i = threadIdx.x; i < n; i += kThreads) d[i] *= scale;
        __syncthreads();
        for (int it = 0; it < bound; ++it) {
          const double beta = dotn(v.Y + (size_t)j * n, d, n, red) / o.ys[j];
          const double c = o.alpha[j] - beta;
          const double* sj = v.S + (size_t)j * n;
          for (size_t i = threadIdx.x; i < n; i += kThreads) d[i] += c * sj[i];
          __syncthreads();
          j = (j + 1) % kM;
        }
        if (threadIdx.x == 0) o.step = 1.0;
        __syncthreads();
        start_ls();
      }
    }
  }
  (void)done;
  __syncthreads();
  if (threadIdx.x == 0) *st = o;
}

__global__ void k_fill_value(double* a, size_t n, double v) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) a[i] = v;
}

__global__ void k_regress_init(RegState* st) {
  RegState o{};
  o.phase = 0;
  *st = o;
}

// solution (original domain) -> x = [log(w) * scale_dic, log(atoms)] (:389-401)
__global__ void k_to_variables(const double* sol, double* x, size_t PK, size_t n, double sd) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    x[i] = i < PK ? log(sol[i]) * sd : log(sol[i]);
}

// x -> solution: exp and normalisation per weight row / atom (:424-448)
__global__ void k_from_variables(const double* x, double* sol, int rows_w, int K, int rows_a, size_t N,
                                 double sd) {
  __shared__ double red[32];
  const int r = blockIdx.x;
  const bool is_w = r < rows_w;
  const size_t len = is_w ? (size_t)K : N;
  const double* in = is_w ? x + (size_t)r * K : x + (size_t)rows_w * K + (size_t)(r - rows_w) * N;
  double* out = is_w ? sol + (size_t)r * K : sol + (size_t)rows_w * K + (size_t)(r - rows_w) * N;
  const double scale = is_w ? 1.0 / sd : 1.0;
  double s = 0;
  for (size_t i = threadIdx.x; i < len; i += blockDim.x) s += exp(in[i] * scale);
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  double tot = 0;
  for (int i = 0; i < (int)(blockDim.x >> 5); ++i) tot += red[i];
  for (size_t i = threadIdx.x; i < len; i += blockDim.x) out[i] = exp(in[i] * scale) / tot;
  (void)rows_a;
}

}  // namespace

int regress_both_dev(wdl_ctx* ctx, int P, int K, int L, int loss_type, double scale_dic, double* solution,
                     const double* observed, int max_iterations, double epsilon, int warm_restart,
                     int* status, double* f_out, int* evaluations, cudaStream_t s) {
  const size_t N = ctx->N, PK = (size_t)P * K, n = PK + (size_t)K * N, PKN = PK * N;
  // state: x, g, xp, gp, d, S, Y, g_eval [n each, S and Y m times], f_eval,
  // the state word; warm restart: b_storage, b_temp [P*K*N]
  const size_t vec = ((n * 8 + 255) / 256) * 256;
  const size_t need = vec * (6 + 2 * kM) + 512 + sizeof(RegState) + (warm_restart ? 2 * PKN * 8 + 512 : 0);
  Arena& A = ctx->lbfgs_arena;
  if (need > A.bytes) {
    WDL_CUDA_TRY(ctx, cudaStreamSynchronize(s));
    if (A.ptr) WDL_CUDA_TRY(ctx, cudaFree(A.ptr));
    A.ptr = nullptr;
    A.bytes = 0;
    WDL_CUDA_TRY(ctx, cudaMalloc(&A.ptr, need));
    A.bytes = need;
  }
  A.reset();
  RegVecs v{};
  v.x = A.take<double>(n);
  v.g = A.take<double>(n);
  v.xp = A.take<double>(n);
  v.gp = A.take<double>(n);
  v.d = A.take<double>(n);
  double* g_eval = A.take<double>(n);
  v.S = A.take<double>(kM * n);
  v.Y = A.take<double>(kM * n);
  double* f_eval = A.take<double>(1);
  RegState* st = A.take<RegState>(1);
  double* b_store = warm_restart ? A.take<double>(PKN) : nullptr;
  double* b_temp = warm_restart ? A.take<double>(PKN) : nullptr;
  v.f_eval = f_eval;
  v.g_eval = g_eval;

  RegParam prm{};
  prm.max_linesearch = 20;  // :367
  prm.epsilon = epsilon;
  prm.ftol = 1e-4;          // liblbfgs defaults (lbfgs.c:124-129)
  prm.wolfe = 0.9;
  prm.min_step = 1e-20;
  prm.max_step = 1e20;
  const int per_run = warm_restart ? 10 : max_iterations;  // :368-371
  const int runs = warm_restart ? max_iterations / 10 : 1;  // :407
  prm.max_iterations = per_run;

  const unsigned grid = grid_for(n, 256, ctx->sm_count);
  k_to_variables<<<grid, 256, 0, s>>>(solution, v.x, PK, n, scale_dic);
  WDL_LAUNCH_CHECK(ctx);
  if (warm_restart) {
    k_fill_value<<<grid_for(PKN, 256, ctx->sm_count), 256, 0, s>>>(b_store, PKN, 1.0);  // :381-384
    WDL_LAUNCH_CHECK(ctx);
  }
  int* h_phase = nullptr;
  WDL_CUDA_TRY(ctx, cudaMallocHost(&h_phase, sizeof(RegState)));
  RegState* h_state = reinterpret_cast<RegState*>(h_phase);
  int rc = WDL_OK, evals = 0, last_status = 0;
  double last_f = 0;
  for (int run = 0; run < runs && rc == WDL_OK; ++run) {
    k_regress_init<<<1, 1, 0, s>>>(st);
    WDL_LAUNCH_CHECK(ctx);
    // at most 1 + max_iterations * max_linesearch evaluations per run
    const long long max_rounds = 1 + (long long)(per_run > 0 ? per_run : 100000) * prm.max_linesearch;
    for (long long round = 0; round < max_rounds; ++round) {
      if ((rc = evaluate_both_dev(ctx, P, K, L, loss_type, scale_dic, v.x, g_eval, (int)n, observed, f_eval,
                                  b_store, b_temp, nullptr, s)))
        break;
      k_regress_step<<<1, kThreads, 0, s>>>(st, v, n, prm);
      WDL_LAUNCH_CHECK(ctx);
      if (cudaMemcpyAsync(h_state, st, sizeof(RegState), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
          cudaStreamSynchronize(s) != cudaSuccess) {
        rc = cuda_error(ctx, cudaGetLastError(), "regress_both round");
        break;
      }
      if ((rc = tc_check_status(ctx))) break;
      if (h_state->phase == 2) break;
    }
    if (rc) break;
    evals += h_state->evals;
    last_status = h_state->status;
    last_f = h_state->f;
    if (warm_restart)  // the run's last scalings start the next run (:411-415)
      WDL_CUDA_TRY(ctx, cudaMemcpyAsync(b_store, b_temp, PKN * 8, cudaMemcpyDeviceToDevice, s));
  }
  if (rc == WDL_OK) {
    k_from_variables<<<P + K, 256, 0, s>>>(v.x, solution, P, K, K, N, scale_dic);
    rc = WDL_OK;
    cudaError_t e = cudaGetLastError();
    ctx->launches++;
    if (e != cudaSuccess) rc = cuda_error(ctx, e, "kernel launch");
  }
  if (rc == WDL_OK) {
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) rc = cuda_error(ctx, e, "regress_both");
  }
  cudaFreeHost(h_phase);
  if (status) *status = last_status;
  if (f_out) *f_out = last_f;
  if (evaluations) *evaluations = evals;
  return rc;
}

}  // namespace wdl
