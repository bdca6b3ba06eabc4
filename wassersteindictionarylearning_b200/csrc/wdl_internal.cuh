// Internal declarations of libwdl_b200: the context, its device workspace and
// the launch helpers shared by the kernel files.  Not part of the ABI.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <functional>
#include <string>
#include <vector>

#include "../../include/wdl.h"

namespace wdl {

// log(1e-250): the value safe_log(x) = log(max(EPSILON, x)) takes at x = 0
// (cpp/loss.h:3-5, EPSILON at cpp/kernels.h:30).  Every positive FP32 number
// exceeds 1e-250, so in FP32 safe_log(x) is log(x) for x > 0 and this constant
// otherwise; in FP64 the floor is applied literally.
constexpr double kLogEpsilon = -575.6462732485114;
constexpr double kEpsilon = 1e-250;

struct Status {
  int code = WDL_OK;
  std::string msg;
};

// Grow-only device arena: one cudaMalloc per high-water mark, reused by every
// call of the same or smaller size.
struct Arena {
  void* ptr = nullptr;
  size_t bytes = 0;
  size_t off = 0;
  void reset() { off = 0; }
  template <typename T>
  T* take(size_t n) {
    off = (off + 255) & ~size_t(255);
    T* p = reinterpret_cast<T*>(static_cast<char*>(ptr) + off);
    off += n * sizeof(T);
    return p;
  }
};

// Size of an arena plan: the same sequence of take<T>(n) calls without memory.
struct ArenaPlan {
  size_t off = 0;
  template <typename T>
  void take(size_t n) {
    off = (off + 255) & ~size_t(255);
    off += n * sizeof(T);
  }
};

struct TcResources;  // tensor-core factor matrices (conv_tc.cu)

}  // namespace wdl

struct wdl_ctx {
  int device = 0;
  int W = 0, H = 0, D = 1;
  int ndim = 2;
  size_t N = 0;
  double gamma = 0;
  int precision = WDL_FP32;
  int domain = WDL_DOMAIN_KERNEL;
  int sm_count = 0;
  cudaStream_t stream = nullptr;

  // Dense Gibbs factor of each axis, G[i][j] = max(EPSILON, exp(-(i-j)^2/gamma)),
  // stored row-major n x n in FP64 and FP32 (cpp/kernels.h:637-640).
  int axis_len[3] = {0, 0, 0};
  // Largest |i - j| whose factor entry is non-zero in FP32, per axis: beyond it
  // (exp(-d^2/gamma) under the FP32 range) the FP32 factor is exactly zero.
  int axis_reach[3] = {0, 0, 0};
  double* G64[3] = {nullptr, nullptr, nullptr};
  float* G32[3] = {nullptr, nullptr, nullptr};

  wdl::Arena arena;  // compute workspace (tape, scratch)
  wdl::Arena io;     // staging of the host-pointer calls
  wdl::Arena lbfgs_arena;  // device L-BFGS state of wdl_regress_both (regress.cu)
  wdl::TcResources* tc = nullptr;
  int* fused_sync = nullptr;  // status block of the last fused-kernel launch (in the arena)
  // Device address of the library's fixed no-allocation scratch array on this
  // context's device, looked up when the context is created (noalloc.cu).
  void* noalloc_scratch = nullptr;
  // Bound on one dependency wait of the fused kernel in seconds (0: the
  // default), and a host-side fault to inject into the next batched launch
  // (wdl_set_wait_limit, wdl_inject_fault).
  double wait_limit_s = 0;
  int inject_fault = 0;

  std::string last_error;
  long long launches = 0;

  bool profiling = false;
  bool autotune = true;  // wdl_set_autotune
  cudaEvent_t ev_a = nullptr, ev_b = nullptr;
  double conv_ms = 0;
  long long conv_launches = 0;
  double conv_images = 0;
  double log_exps = 0;                 // exps the log-domain passes executed (profiling)
  unsigned long long* d_taps = nullptr;  // device counter of those exps
  int trace_level = 0;                    // 2: per-phase device trace of the fused kernel
  unsigned long long* d_trace = nullptr;  // [27] accumulated ns / counts

  // Replayable evaluations of the multi-launch (CUDA-core) path: a call whose
  // sizes, pointers, stream and workspace match a previous call replays that
  // call's launches as one CUDA graph (sinkhorn.cu).
  struct GraphEntry {
    unsigned long long key[20];
    int seen = 0;
    cudaGraphExec_t exec = nullptr;
    long long launches = 0;
  };
  std::vector<GraphEntry> graphs;

  // Autotuned launch shapes (conv_simt.cu): key -> chosen variant.
  struct TuneEntry {
    long long key[6];
    int choice = 0;
    float ms = 0;
  };
  std::vector<TuneEntry> tuned;
};

namespace wdl {

int set_error(wdl_ctx* ctx, int code, const std::string& msg);
// WDL_AUTOTUNE=0 in the environment turns the launch-shape autotuner off.
bool autotune_enabled();
int cuda_error(wdl_ctx* ctx, cudaError_t e, const char* where);
int ensure_arena(wdl_ctx* ctx, size_t bytes);
// Looks up the no-allocation scratch array's address on the current device
// into ctx->noalloc_scratch (noalloc.cu); called by wdl_create.
int noalloc_attach(wdl_ctx* ctx);

#define WDL_CUDA_TRY(ctx, expr)                                    \
  do {                                                             \
    cudaError_t _e = (expr);                                       \
    if (_e != cudaSuccess) return ::wdl::cuda_error(ctx, _e, #expr); \
  } while (0)

#define WDL_LAUNCH_CHECK(ctx)                                                   \
  do {                                                                          \
    (ctx)->launches++;                                                          \
    cudaError_t _e = cudaGetLastError();                                        \
    if (_e != cudaSuccess) return ::wdl::cuda_error(ctx, _e, "kernel launch");  \
  } while (0)

inline unsigned grid_for(size_t n, int block, int sm_count, int per_sm = 8) {
  size_t g = (n + block - 1) / block;
  size_t cap = (size_t)sm_count * per_sm;
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return (unsigned)g;
}

// ---- separable operator (conv_simt.cu / conv_tc.cu) ----------------------------
// out_v = G (*) in_v for nimg stacked images of the context's grid.  in and out
// must not alias; tmp holds nimg*N elements.
int conv_stack_f32(wdl_ctx* ctx, const float* in, float* out, float* tmp, size_t nimg,
                   cudaStream_t s);
int conv_stack_f64(wdl_ctx* ctx, const double* in, double* out, double* tmp, size_t nimg,
                   cudaStream_t s);
int conv_stack_simt_f32(wdl_ctx* ctx, const float* in, float* out, float* tmp, size_t nimg,
                        cudaStream_t s);
// Log-sum-exp operator; signs (one byte per element, 1 = non-negative) are read
// from in_sign and written to out_sign when non-null.  With sub_from non-null
// (unsigned only) the last pass also writes sub_out[i] = sub_from[i mod
// sub_period] - out[i] for every element i of the nimg images.
int log_conv_stack_f32(wdl_ctx* ctx, const float* in, float* out, float* tmp, size_t nimg,
                       const uint8_t* in_sign, uint8_t* out_sign, uint8_t* tmp_sign,
                       cudaStream_t s, const float* sub_from = nullptr, float* sub_out = nullptr,
                       size_t sub_period = 0);
int log_conv_stack_f64(wdl_ctx* ctx, const double* in, double* out, double* tmp, size_t nimg,
                       const uint8_t* in_sign, uint8_t* out_sign, uint8_t* tmp_sign,
                       cudaStream_t s, const double* sub_from = nullptr, double* sub_out = nullptr,
                       size_t sub_period = 0);

template <typename T>
inline int conv_stack(wdl_ctx* ctx, const T* in, T* out, T* tmp, size_t nimg, cudaStream_t s);
template <>
inline int conv_stack<float>(wdl_ctx* ctx, const float* in, float* out, float* tmp, size_t nimg,
                             cudaStream_t s) {
  return conv_stack_f32(ctx, in, out, tmp, nimg, s);
}
template <>
inline int conv_stack<double>(wdl_ctx* ctx, const double* in, double* out, double* tmp,
                              size_t nimg, cudaStream_t s) {
  return conv_stack_f64(ctx, in, out, tmp, nimg, s);
}

template <typename T>
inline int log_conv_stack(wdl_ctx* ctx, const T* in, T* out, T* tmp, size_t nimg,
                          const uint8_t* in_sign, uint8_t* out_sign, uint8_t* tmp_sign,
                          cudaStream_t s, const T* sub_from = nullptr, T* sub_out = nullptr,
                          size_t sub_period = 0);
template <>
inline int log_conv_stack<float>(wdl_ctx* ctx, const float* in, float* out, float* tmp,
                                 size_t nimg, const uint8_t* is, uint8_t* os, uint8_t* ts,
                                 cudaStream_t s, const float* sf, float* so, size_t sp) {
  return log_conv_stack_f32(ctx, in, out, tmp, nimg, is, os, ts, s, sf, so, sp);
}
template <>
inline int log_conv_stack<double>(wdl_ctx* ctx, const double* in, double* out, double* tmp,
                                  size_t nimg, const uint8_t* is, uint8_t* os, uint8_t* ts,
                                  cudaStream_t s, const double* sf, double* so, size_t sp) {
  return log_conv_stack_f64(ctx, in, out, tmp, nimg, is, os, ts, s, sf, so, sp);
}

// Tensor-core resources (conv_tc.cu).
int tc_init(wdl_ctx* ctx);
void tc_free(wdl_ctx* ctx);
// Reads and clears the status word the tensor-core kernels set when a bounded
// wait gives up (WDL_ERR_TIMEOUT); WDL_OK otherwise.
int tc_check_status(wdl_ctx* ctx);
// regress_both with the L-BFGS on the device (regress.cu); solution and
// observed are device pointers.
int regress_both_dev(wdl_ctx* ctx, int P, int K, int L, int loss_type, double scale_dic, double* solution,
                     const double* observed, int max_iterations, double epsilon, int warm_restart,
                     int* status, double* f_out, int* evaluations, cudaStream_t s);
bool tc_supported(const wdl_ctx* ctx);
// The context has the fused Sinkhorn kernel (tensor-core precision, 2-D, sides <= 128).
bool tc_fused(const wdl_ctx* ctx);
// Tensor-core axis passes (conv_tc_axis.cu): any tensor-core context.
int tc_axis_init(wdl_ctx* ctx, uint8_t* (&blocks)[3]);
int conv_stack_tc_axes(wdl_ctx* ctx, const float* in, float* out, float* tmp, size_t nimg,
                       uint8_t* const (&blocks)[3], int* err, cudaStream_t s);

// Fused persistent tensor-core Sinkhorn kernel (sinkhorn_tc.cu).
// One problem of a fused launch: P histograms on one W x H grid (sides <= 128)
// against K atoms, L iterations.  Pointers are device buffers of this problem.
struct SkProblem {
  int W, H, Wp, Hp, K, L, P, loss_type;
  int fwd_only;   // forward only (barycenters): two tape slots, no loss
  int need_dic;   // run the dictionary recursion (atom gradient); 0 = weights only
  int vec;        // rows are 16-byte aligned (W % 4 == 0)
  uint32_t cpr, cpr_magic;  // operand chunks per row, ceil(2^32 / cpr)
  size_t N;
  const float* atoms;    // [K][N]
  const float* lam;      // [P][K]
  const double* obs;     // [P][N]
  const float* b0;       // [P][K][N] or null (ones)
  float* cb;             // [slots][P][K][N]   conv_b tape
  float* phi;            // [slots][P][K][N]   phi tape
  float* acc;            // [slots][P][N]      sum_k lambda_k safe_log(phi_k): bary = exp(acc)
  float *nb, *gwb;       // [2][P][N]          reverse-pass messages, by step parity
  float *v, *r, *gdic;   // [P][K][N]
  double* dot;           // [P][K]
  double* loss;          // [P]
  int* sync;             // done_fwd[P], bary_ready[P], done_bwd[P], msg_ready[P], range[P]
};

struct SkArgs {
  const float* G;        // factor matrix of the launch's gamma, Gn x Gn
  int Gn, nprobs;
  const SkProblem* probs;     // device array [nprobs]
  const int4* items;          // (problem, type, step, pk) per work item, or null: problem 0
  long long total;            // work items
  double apps;                // operator applications the items perform (for profiling)
  int* sync;                  // work counter, error word
  unsigned long long* trace;  // [3 item types][8 phases + 1 count] ns, or null
  unsigned long long dep_wait_ns;  // bound on one dependency wait
};
// Host helpers of the fused launch.
void sk_fill_geometry(SkProblem& pr, int W, int H, bool split_bf16);
size_t sk_problem_items(const SkProblem& pr);
double sk_problem_applications(const SkProblem& pr);
int sinkhorn_tc_launch(wdl_ctx* ctx, SkArgs& a, cudaStream_t s);
int sinkhorn_tc_status(wdl_ctx* ctx, int* sync_dev);

// ---- many problems per launch (batch.cu, fit.cu) ---------------------------------
struct BatchBuf {  // one problem's device buffers inside the arena
  double *atoms64, *lam64, *dot, *loss, *obs, *in_atoms, *in_w, *out_la, *out_loss, *out_bary,
      *out_dic;
  float *atoms, *lam, *cb, *phi, *acc, *nb, *gwb, *v, *r, *gdic;
  int* sync;
};
struct BatchPlan {
  int nprob = 0;
  char* base = nullptr;               // arena base the offsets refer to
  std::vector<BatchBuf> buf;
  std::vector<SkProblem> prs;
  size_t probs = 0, gsync = 0, zero_b = 0, zero_e = 0, in_b = 0, in_e = 0, out_b = 0, out_e = 0;
  size_t rows_off = 0, outj_off = 0, items_off = 0, extra_off = 0;
  size_t n_outjobs = 0, n_items_all = 0;
  int* sync = nullptr;                // work counter, error word of the fused launch
};
// Validates, lays out and uploads every problem (inputs normalised on the
// device); reserves extra_bytes at plan.extra_off for the caller.
int batch_prepare(wdl_ctx* ctx, const wdl_problem* pb, int nprob, size_t extra_bytes, BatchPlan& bp,
                  cudaStream_t s);
// Work items by round (every problem's forward iteration r, then its reverse
// step 2L-r), for the histograms whose flag in `active` is set (flattened
// problem by problem; null = all).
void batch_items(const BatchPlan& bp, const std::vector<uint8_t>* active, std::vector<int4>& items);
// Clears the accumulated buffers and launches the fused kernel over the first
// n_items entries of the item table at plan.items_off.
int batch_launch(wdl_ctx* ctx, BatchPlan& bp, size_t n_items, cudaStream_t s);

// Hot path entry points (sinkhorn.cu); all pointers are device pointers.
int gradient_both_dev(wdl_ctx* ctx, int P, int K, int L, int loss_type, const double* atoms,
                      const double* weights, const double* observed, const double* b_init,
                      double* result_la, double* result_dic, double* bary, double* loss,
                      double* b_last, cudaStream_t s, bool normalise);
int evaluate_both_dev(wdl_ctx* ctx, int P, int K, int L, int loss_type, double scale_dic,
                      const double* x, double* g, int n, const double* observed, double* f,
                      const double* b_storage, double* b_last, double* bary, cudaStream_t s);
int barycenter_dev(wdl_ctx* ctx, int P, int K, int L, const double* atoms, const double* weights,
                   double* bary, cudaStream_t s);
size_t eval_bytes(const wdl_ctx* ctx, int P, int K, int L);
// Runs `run` (a fixed sequence of launches on s) eagerly the first time a key
// is seen, captures it into a CUDA graph the second time and replays the graph
// afterwards (sinkhorn.cu); inside a caller's capture it just runs.  The key
// must name every size, pointer and parameter the launches depend on.
int replay_or_run(wdl_ctx* ctx, const unsigned long long (&key)[20], cudaStream_t s,
                  const std::function<int()>& run);
size_t barycenter_bytes(const wdl_ctx* ctx, int P, int K);

}  // namespace wdl
