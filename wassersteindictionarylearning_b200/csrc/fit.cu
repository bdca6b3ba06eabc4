// wdl_fit_weights: batched weight fitting (projection onto fixed dictionaries)
// with the L-BFGS outer loop on the device.
//
// The reference fits weights with liblbfgs on the host around evaluate_both
// (regress_both, cpp/inverseWasserstein.h:362-423; lbfgs.c:256-654 with the
// strong-Wolfe backtracking line search of lbfgs.c:772-867).  Here every
// histogram of every problem is one optimisation whose state (x, g, the
// previous point, the direction, m = 6 correction pairs) lives in device
// memory.  One round is: the fused kernel evaluates every active histogram at
// its current trial point (many problems per launch, wdl_batch_run's layout),
// then k_fit_round consumes each loss and weight gradient and advances that
// optimisation's state machine to its next trial point.  The round is captured
// once in a CUDA graph and replayed; the host only looks at the done flags
// every few rounds to drop finished histograms from the item table.
//
// Variables: x in R^K per histogram, weights = softmax(x) (the reference's
// exp_weight transform with scaleDictionary 1 followed by the normalisation
// by the sum, cpp/inverseWasserstein.h:1000-1020); gradient =
// (la - <w, la>) * w, the projection and chain rule of evaluate_both
// (:1092-1097, :1124-1133).
#include <cmath>
#include <cstring>
#include <vector>

#include "lbfgs_dev.cuh"
#include "wdl_internal.cuh"

namespace wdl {
namespace {

using namespace lbdev;

struct LbOpt {
  LbState s;
  double* v;            // state vectors (pool_doubles(K))
  double* lam64;        // the weights the fused kernel evaluates ([K], FP64 and FP32)
  float* lam32;
  const double* dot;    // weight gradient of that evaluation ([K], raw resultLa)
  const double* loss;   // its loss
};

__global__ void k_fit_init(LbOpt* opts, int n, const double* x0s) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  LbOpt o = opts[i];
  double* x = o.v;
  for (int k = 0; k < o.s.K; ++k) x[k] = x0s ? x0s[(size_t)i * 64 + k] : 0.0;
  softmax_weights(x, o.s.K, o.lam64, o.lam32);
}

// One optimisation step per histogram: consume the evaluation at the current
// trial point, move to the next trial point (or finish).  A non-finite
// evaluation means the kernel domain overflowed at this point.
__global__ void k_fit_round(LbOpt* opts, int n, LbParam prm, const int* fused_sync, int* sticky,
                            uint8_t* done) {
  __shared__ int s_err;
  if (threadIdx.x == 0) s_err = *(volatile const int*)(fused_sync + 1);
  __syncthreads();
  if (s_err) {  // the evaluation is incomplete: consume nothing
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicExch(sticky, s_err);
    return;
  }
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  LbOpt o = opts[i];
  if (o.s.phase == 2) return;
  lbfgs_advance(o.s, o.v, o.loss[0], o.dot, o.lam64, o.lam32, prm, WDL_FIT_OVERFLOW);
  opts[i] = o;
  done[i] = o.s.phase == 2 ? 1 : 0;
}

// k_fit_round with the L-BFGS settings read from device memory, so that a
// recorded round does not depend on them.
__global__ void k_fit_round_dp(LbOpt* opts, int n, const LbParam* prm, uint8_t* done) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  LbOpt o = opts[i];
  if (o.s.phase == 2) return;
  const LbParam pv = *prm;
  lbfgs_advance(o.s, o.v, o.loss[0], o.dot, o.lam64, o.lam32, pv, WDL_FIT_OVERFLOW);
  opts[i] = o;
  done[i] = o.s.phase == 2 ? 1 : 0;
}

struct FitOut {
  double w[64];
  double loss;
  int status, evals;
};

__global__ void k_fit_outputs(const LbOpt* opts, int n, FitOut* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const LbOpt o = opts[i];
  softmax_weights(o.v, o.s.K, out[i].w, nullptr);
  out[i].loss = o.s.phase == 2 ? o.s.fret : o.s.f;
  out[i].status = o.s.phase == 2 ? o.s.status : kMaximumIteration;
  out[i].evals = o.s.evals;
}

inline size_t a256(size_t b) { return (b + 255) & ~size_t(255); }

}  // namespace
}  // namespace wdl

using namespace wdl;

extern "C" int wdl_fit_weights(wdl_ctx* ctx, const wdl_fit_problem* fp, int nprob, int max_iterations,
                               double epsilon) {
  if (!ctx) return WDL_ERR_INVALID_ARG;
  if (!fp || nprob < 1 || max_iterations < 0 || !(epsilon >= 0))
    return set_error(ctx, WDL_ERR_INVALID_ARG, "bad arguments");
  if (cudaSetDevice(ctx->device) != cudaSuccess) return set_error(ctx, WDL_ERR_CUDA, "cudaSetDevice failed");
  cudaStream_t s = ctx->stream;
  // The batch layout with weights-only problems; the starting weights are
  // placeholders that k_fit_init overwrites.
  std::vector<wdl_problem> pb(nprob);
  size_t nopt = 0, pool = 0, max_pk = 0;
  for (int q = 0; q < nprob; ++q) {
    const wdl_fit_problem& f = fp[q];
    if (f.K < 1 || f.K > 64 || f.P < 1 || !f.atoms || !f.observed || !f.weights || !f.loss ||
        !f.status || !f.evaluations)
      return set_error(ctx, WDL_ERR_INVALID_ARG, "fit problem " + std::to_string(q) + ": bad sizes or pointers");
    nopt += f.P;
    pool += (size_t)f.P * pool_doubles(f.K);
    if ((size_t)f.P * f.K > max_pk) max_pk = (size_t)f.P * f.K;
  }
  std::vector<double> ones(max_pk, 1.0);
  for (int q = 0; q < nprob; ++q) {
    const wdl_fit_problem& f = fp[q];
    wdl_problem& w = pb[q];
    w = wdl_problem{};
    w.W = f.W;
    w.H = f.H;
    w.K = f.K;
    w.L = f.L;
    w.P = f.P;
    w.loss_type = f.loss_type;
    w.mode = WDL_MODE_WEIGHTS;
    w.atoms = f.atoms;
    w.weights = ones.data();
    w.observed = f.observed;
  }
  // extra region: optimiser table, state pool, starting points, outputs, flags
  const size_t off_opts = 0;
  const size_t off_pool = a256(off_opts + nopt * sizeof(LbOpt));
  const size_t off_x0 = a256(off_pool + pool * sizeof(double));
  const size_t off_out = a256(off_x0 + nopt * 64 * sizeof(double));
  const size_t off_done = a256(off_out + nopt * sizeof(FitOut));
  const size_t off_sticky = a256(off_done + nopt);
  const size_t extra = off_sticky + 256;
  BatchPlan bp;
  int rc;
  if ((rc = batch_prepare(ctx, pb.data(), nprob, extra, bp, s))) return rc;
  char* ex = bp.base + bp.extra_off;
  LbOpt* d_opts = reinterpret_cast<LbOpt*>(ex + off_opts);
  double* d_pool = reinterpret_cast<double*>(ex + off_pool);
  double* d_x0 = reinterpret_cast<double*>(ex + off_x0);
  FitOut* d_out = reinterpret_cast<FitOut*>(ex + off_out);
  uint8_t* d_done = reinterpret_cast<uint8_t*>(ex + off_done);
  int* d_sticky = reinterpret_cast<int*>(ex + off_sticky);

  std::vector<LbOpt> opts(nopt);
  std::vector<double> x0(nopt * 64, 0.0);
  bool any_x0 = false;
  {
    size_t i = 0, po = 0;
    for (int q = 0; q < nprob; ++q) {
      const wdl_fit_problem& f = fp[q];
      const BatchBuf& b = bp.buf[q];
      for (int p = 0; p < f.P; ++p, ++i) {
        LbOpt o{};
        o.s.K = f.K;
        o.v = d_pool + po;
        po += pool_doubles(f.K);
        o.lam64 = b.lam64 + (size_t)p * f.K;
        o.lam32 = b.lam + (size_t)p * f.K;
        o.dot = b.dot + (size_t)p * f.K;
        o.loss = b.loss + p;
        opts[i] = o;
        if (f.x0) {
          any_x0 = true;
          for (int k = 0; k < f.K; ++k) x0[i * 64 + k] = f.x0[(size_t)p * f.K + k];
        }
      }
    }
  }
  WDL_CUDA_TRY(ctx, cudaMemcpyAsync(d_opts, opts.data(), nopt * sizeof(LbOpt), cudaMemcpyHostToDevice, s));
  if (any_x0) WDL_CUDA_TRY(ctx, cudaMemcpyAsync(d_x0, x0.data(), x0.size() * sizeof(double), cudaMemcpyHostToDevice, s));
  WDL_CUDA_TRY(ctx, cudaMemsetAsync(d_done, 0, nopt, s));
  WDL_CUDA_TRY(ctx, cudaMemsetAsync(d_sticky, 0, sizeof(int), s));
  const unsigned og = (unsigned)((nopt + 127) / 128);
  k_fit_init<<<og, 128, 0, s>>>(d_opts, (int)nopt, any_x0 ? d_x0 : nullptr);
  WDL_LAUNCH_CHECK(ctx);

  LbParam prm{max_iterations, 20, epsilon, 1e-4, 0.9, 1e-20, 1e20};
  // every trial is one round; a histogram needs at most (1 + max_linesearch)
  // rounds per iteration
  const long long max_rounds = (long long)(max_iterations > 0 ? max_iterations : 1000) * (prm.max_linesearch + 1) + 2;
  const int chunk = 4;  // rounds replayed between looks at the done flags
  std::vector<uint8_t> active(nopt, 1), h_done(nopt, 0);
  std::vector<int4> items;
  const bool prof = ctx->profiling;
  const int trace = ctx->trace_level;
  ctx->profiling = false;  // no event synchronisation inside a capture
  ctx->trace_level = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  long long rounds = 0;
  int kernels_per_round = 0;
  auto release = [&]() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    exec = nullptr;
    graph = nullptr;
  };
  auto restore = [&]() {
    ctx->profiling = prof;
    ctx->trace_level = trace;
  };
  rc = WDL_OK;
  while (rounds < max_rounds) {
    size_t n_active = 0;
    for (uint8_t a : active) n_active += a;
    if (!n_active) break;
    if (!exec) {  // item table of the active histograms, one round captured
      batch_items(bp, &active, items);
      cudaError_t e = cudaMemcpyAsync(bp.base + bp.items_off, items.data(), items.size() * sizeof(int4),
                                      cudaMemcpyHostToDevice, s);
      if (e == cudaSuccess) e = cudaStreamSynchronize(s);
      if (e != cudaSuccess) { rc = cuda_error(ctx, e, "item table upload"); break; }
      const long long l0 = ctx->launches;
      e = cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed);
      if (e != cudaSuccess) { rc = cuda_error(ctx, e, "cudaStreamBeginCapture"); break; }
      int lr = batch_launch(ctx, bp, items.size(), s);
      if (!lr) {
        k_fit_round<<<og, 128, 0, s>>>(d_opts, (int)nopt, prm, bp.sync, d_sticky, d_done);
        ctx->launches++;
      }
      e = cudaStreamEndCapture(s, &graph);
      if (lr) { rc = lr; break; }
      if (e != cudaSuccess) { rc = cuda_error(ctx, e, "cudaStreamEndCapture"); break; }
      e = cudaGraphInstantiate(&exec, graph, 0);
      if (e != cudaSuccess) { rc = cuda_error(ctx, e, "cudaGraphInstantiate"); break; }
      kernels_per_round = (int)(ctx->launches - l0);
      ctx->launches = l0;
    }
    cudaError_t e = cudaSuccess;
    for (int r = 0; r < chunk && rounds < max_rounds && e == cudaSuccess; ++r, ++rounds) {
      e = cudaGraphLaunch(exec, s);
      ctx->launches += kernels_per_round;
    }
    int sticky = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(h_done.data(), d_done, nopt, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&sticky, d_sticky, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) { rc = cuda_error(ctx, e, "fit round"); break; }
    if (sticky) { rc = set_error(ctx, sticky, "fused tensor-core kernel: a bounded wait timed out"); break; }
    bool changed = false;
    for (size_t i = 0; i < nopt; ++i)
      if (active[i] && h_done[i]) {
        active[i] = 0;
        changed = true;
      }
    if (changed) release();
  }
  release();
  restore();
  if (rc) return rc;
  k_fit_outputs<<<og, 128, 0, s>>>(d_opts, (int)nopt, d_out);
  WDL_LAUNCH_CHECK(ctx);
  std::vector<FitOut> h_out(nopt);
  WDL_CUDA_TRY(ctx, cudaMemcpyAsync(h_out.data(), d_out, nopt * sizeof(FitOut), cudaMemcpyDeviceToHost, s));
  WDL_CUDA_TRY(ctx, cudaStreamSynchronize(s));
  size_t i = 0;
  for (int q = 0; q < nprob; ++q) {
    const wdl_fit_problem& f = fp[q];
    for (int p = 0; p < f.P; ++p, ++i) {
      for (int k = 0; k < f.K; ++k) f.weights[(size_t)p * f.K + k] = h_out[i].w[k];
      f.loss[p] = h_out[i].loss;
      f.status[p] = h_out[i].status;
      f.evaluations[p] = h_out[i].evals;
    }
  }
  return WDL_OK;
}

// wdl_fit_weights_operator: the fits of wdl_fit_weights for P histograms on the
// context's own grid and evaluation path.  Round r evaluates the P histograms
// at their current trial points (gradient_both_dev, weights only: the weight
// gradient resultLa and the loss) and k_fit_round advances every optimisation.
// The first round runs eagerly (it sizes the context's workspace); the next
// ones are captured once and replayed.
extern "C" int wdl_fit_weights_operator(wdl_ctx* ctx, int P, int K, int L, int loss_type, const double* atoms,
                                        const double* observed, const double* x0, int max_iterations,
                                        double epsilon, double* weights, double* loss, int* status,
                                        int* evaluations) {
  if (!ctx) return WDL_ERR_INVALID_ARG;
  if (P < 1 || K < 1 || K > 64 || L < 1 || max_iterations < 0 || !(epsilon >= 0) || !atoms || !observed ||
      !weights || !loss || !status || !evaluations)
    return set_error(ctx, WDL_ERR_INVALID_ARG, "bad sizes or NULL required pointer");
  if (loss_type < WDL_LOSS_TV || loss_type > WDL_LOSS_KL)
    return set_error(ctx, WDL_ERR_INVALID_ARG, "loss_type must be 1..4");
  if (tc_fused(ctx) && ctx->domain == WDL_DOMAIN_KERNEL && loss_type != WDL_LOSS_WASSERSTEIN)
    return set_error(ctx, WDL_ERR_UNSUPPORTED, "fused tensor-core context: use wdl_fit_weights");
  if (cudaSetDevice(ctx->device) != cudaSuccess) return set_error(ctx, WDL_ERR_CUDA, "cudaSetDevice failed");
  cudaStream_t s = ctx->stream;
  const size_t N = ctx->N, KN = (size_t)K * N, PK = (size_t)P * K, PN = (size_t)P * N;
  // device layout: atoms, observed, weights under evaluation, resultLa, loss,
  // optimiser table and state pool, starting points, outputs, done flags, a
  // zeroed word pair standing for the fused kernel's error flag
  ArenaPlan plan;
  plan.take<double>(KN);
  plan.take<double>(PN);
  plan.take<double>(PK);
  plan.take<double>(PK);
  plan.take<double>(P);
  plan.take<LbOpt>(P);
  plan.take<double>((size_t)P * pool_doubles(K));
  plan.take<double>((size_t)P * 64);
  plan.take<FitOut>(P);
  plan.take<uint8_t>(P);
  plan.take<LbParam>(1);
  Arena& A = ctx->lbfgs_arena;
  if (plan.off + 256 > A.bytes) {
    WDL_CUDA_TRY(ctx, cudaStreamSynchronize(s));
    if (A.ptr) WDL_CUDA_TRY(ctx, cudaFree(A.ptr));
    A.ptr = nullptr;
    A.bytes = 0;
    WDL_CUDA_TRY(ctx, cudaMalloc(&A.ptr, plan.off + 256));
    A.bytes = plan.off + 256;
  }
  A.reset();
  double* d_atoms = A.take<double>(KN);
  double* d_obs = A.take<double>(PN);
  double* d_lam = A.take<double>(PK);
  double* d_la = A.take<double>(PK);
  double* d_loss = A.take<double>(P);
  LbOpt* d_opts = A.take<LbOpt>(P);
  double* d_pool = A.take<double>((size_t)P * pool_doubles(K));
  double* d_x0 = A.take<double>((size_t)P * 64);
  FitOut* d_out = A.take<FitOut>(P);
  uint8_t* d_done = A.take<uint8_t>(P);
  LbParam* d_prm = A.take<LbParam>(1);
  std::vector<LbOpt> opts(P);
  std::vector<double> h_x0((size_t)P * 64, 0.0);
  for (int p = 0; p < P; ++p) {
    LbOpt o{};
    o.s.K = K;
    o.v = d_pool + (size_t)p * pool_doubles(K);
    o.lam64 = d_lam + (size_t)p * K;
    o.lam32 = nullptr;
    o.dot = d_la + (size_t)p * K;
    o.loss = d_loss + p;
    opts[p] = o;
    if (x0)
      for (int k = 0; k < K; ++k) h_x0[(size_t)p * 64 + k] = x0[(size_t)p * K + k];
  }
  WDL_CUDA_TRY(ctx, cudaMemcpyAsync(d_atoms, atoms, KN * 8, cudaMemcpyHostToDevice, s));
  WDL_CUDA_TRY(ctx, cudaMemcpyAsync(d_obs, observed, PN * 8, cudaMemcpyHostToDevice, s));
  WDL_CUDA_TRY(ctx, cudaMemcpyAsync(d_opts, opts.data(), P * sizeof(LbOpt), cudaMemcpyHostToDevice, s));
  if (x0) WDL_CUDA_TRY(ctx, cudaMemcpyAsync(d_x0, h_x0.data(), h_x0.size() * 8, cudaMemcpyHostToDevice, s));
  WDL_CUDA_TRY(ctx, cudaMemsetAsync(d_done, 0, P, s));
  const LbParam prm{max_iterations, 20, epsilon, 1e-4, 0.9, 1e-20, 1e20};
  WDL_CUDA_TRY(ctx, cudaMemcpyAsync(d_prm, &prm, sizeof(prm), cudaMemcpyHostToDevice, s));
  const unsigned og = (unsigned)((P + 127) / 128);
  k_fit_init<<<og, 128, 0, s>>>(d_opts, P, x0 ? d_x0 : nullptr);
  WDL_LAUNCH_CHECK(ctx);
  const long long max_rounds = (long long)(max_iterations > 0 ? max_iterations : 1000) * (prm.max_linesearch + 1) + 2;
  // one round: the evaluation of every histogram, then one step of each fit
  auto round = [&]() -> int {
    int rc = gradient_both_dev(ctx, P, K, L, loss_type, d_atoms, d_lam, d_obs, nullptr, d_la, nullptr, nullptr,
                               d_loss, nullptr, s, true);
    if (rc) return rc;
    k_fit_round_dp<<<og, 128, 0, s>>>(d_opts, P, d_prm, d_done);
    WDL_LAUNCH_CHECK(ctx);
    return WDL_OK;
  };
  // Rounds go through the context's graph cache: the workspace is sized first,
  // so a later call with the same sizes (whatever its L-BFGS settings, which
  // the round reads from device memory) replays the same recorded round from
  // its first round on.
  int rc = ensure_arena(ctx, eval_bytes(ctx, P, K, L));
  if (rc) return rc;
  const unsigned long long key[20] = {
      3ull, (unsigned long long)P, (unsigned long long)K, (unsigned long long)L, (unsigned long long)loss_type,
      0ull, 0ull, (unsigned long long)(uintptr_t)A.ptr,
      (unsigned long long)A.bytes, (unsigned long long)(uintptr_t)s, (unsigned long long)(uintptr_t)ctx->arena.ptr,
      (unsigned long long)ctx->arena.bytes, 0ull, 0ull, 0ull, 0ull, 0ull, 0ull, 0ull, 0ull};
  const int chunk = 4;  // rounds between looks at the done flags
  std::vector<uint8_t> h_done(P, 0);
  long long rounds = 0;
  while (rounds < max_rounds) {
    for (int r = 0; r < chunk && rounds < max_rounds; ++r, ++rounds)
      if ((rc = replay_or_run(ctx, key, s, round)) != WDL_OK) return rc;
    WDL_CUDA_TRY(ctx, cudaMemcpyAsync(h_done.data(), d_done, P, cudaMemcpyDeviceToHost, s));
    WDL_CUDA_TRY(ctx, cudaStreamSynchronize(s));
    bool all = true;
    for (uint8_t d : h_done) all = all && d;
    if (all) break;
  }
  k_fit_outputs<<<og, 128, 0, s>>>(d_opts, P, d_out);
  WDL_LAUNCH_CHECK(ctx);
  std::vector<FitOut> h_out(P);
  WDL_CUDA_TRY(ctx, cudaMemcpyAsync(h_out.data(), d_out, P * sizeof(FitOut), cudaMemcpyDeviceToHost, s));
  WDL_CUDA_TRY(ctx, cudaStreamSynchronize(s));
  for (int p = 0; p < P; ++p) {
    for (int k = 0; k < K; ++k) weights[(size_t)p * K + k] = h_out[p].w[k];
    loss[p] = h_out[p].loss;
    status[p] = h_out[p].status == WDL_FIT_OVERFLOW ? WDL_ERR_NONFINITE : h_out[p].status;
    evaluations[p] = h_out[p].evals;
  }
  return WDL_OK;
}
