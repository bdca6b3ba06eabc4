/* wdl.h — C ABI of the B200 Sinkhorn-barycenter library (libwdl_b200.so).
 *
 * Drop-in boundary for the hot path of Wasserstein dictionary learning
 * (reference: matthieuheitz/WassersteinDictionaryLearning, cpp/).  Everything
 * below takes plain pointers and sizes; no exception crosses it; every call
 * returns an int status (WDL_OK = 0, negative WDL_ERR_* on failure, described
 * by wdl_strerror / wdl_last_error).  There is no CPU fallback: without a
 * usable sm_100 device, wdl_create fails with WDL_ERR_NO_DEVICE.
 *
 * Data layout is the reference's: an image of N = W*H*D pixels is row-major
 * with x fastest (index y*W + x, 3-D z*W*H + y*W + x); K images are stacked
 * with stride N; P histograms are stacked with stride N; weights are [P][K];
 * the L-BFGS vector is x = [P*K scaled log-weights, K*N log-atoms]
 * (cpp/main_dictionary_learning.cpp:139-159, cpp/inverseWasserstein.h:389-401).
 *
 * Host-pointer calls copy in, run on the context's stream and copy out before
 * returning.  *_device calls take device pointers and a cudaStream_t passed as
 * void* (NULL = the context's stream) and return without synchronising.
 * One host thread per context; a context is not safe for concurrent calls.
 */
#ifndef WDL_H
#define WDL_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define WDL_ABI_VERSION 1

/* Status codes.  The reference has no error channel of its own (convolutions
 * return void); its only codes are liblbfgs' (cpp/lbfgs/lbfgs.h:74-147), which
 * wdl_lbfgs_* reuse with the same values. */
enum {
  WDL_OK = 0,
  WDL_ERR_INVALID_ARG = -1,
  WDL_ERR_CUDA = -2,
  WDL_ERR_OUT_OF_MEMORY = -3,
  WDL_ERR_UNSUPPORTED = -4,
  WDL_ERR_NONFINITE = -5,   /* a loss or gradient came out NaN/Inf */
  WDL_ERR_TIMEOUT = -6,     /* a bounded device or host wait gave up */
  WDL_ERR_ADMISSION = -7,   /* serving: request larger than the HBM budget */
  WDL_ERR_NO_DEVICE = -8,
  WDL_ERR_BUSY = -9
};

/* Arithmetic of the separable convolutions.  FP32/TF32/SPLIT_BF16 keep the
 * Sinkhorn scalings, tape and elementwise work in FP32 and reduce loss and
 * gradients over grid and batch in FP64; FP64 runs everything in FP64 and
 * keeps the reference's EPSILON = 1e-250 floor (cpp/kernels.h:30). */
typedef enum {
  WDL_FP32 = 0,        /* CUDA-core FP32 FMA                                   */
  WDL_TF32 = 1,        /* tcgen05 kind::tf32, FP32 accumulate                  */
  WDL_SPLIT_BF16 = 2,  /* tcgen05 kind::f16, hi+lo BF16, 3 products, FP32 acc  */
  WDL_FP64 = 3         /* CUDA-core FP64                                       */
} wdl_precision;

typedef enum {
  WDL_DOMAIN_KERNEL = 0, /* scalings as values (compute_gradient_both)              */
  WDL_DOMAIN_LOG = 1     /* scalings as logs (compute_gradient_both_log_signArray)  */
} wdl_domain;

/* Loss indices follow the app's -l flag (cpp/main_dictionary_learning.cpp:189-197). */
typedef enum {
  WDL_LOSS_TV = 1,
  WDL_LOSS_QUADRATIC = 2,
  WDL_LOSS_WASSERSTEIN = 3,
  WDL_LOSS_KL = 4
} wdl_loss;

typedef struct wdl_ctx wdl_ctx;

/* Library and error strings. */
int wdl_abi_version(void);
const char* wdl_strerror(int status);
/* Detail of the last failing call on ctx (or of the last failing wdl_create
 * when ctx is NULL). */
const char* wdl_last_error(const wdl_ctx* ctx);

/* Context for one grid (W, H, D; D = 1 for 2-D) and regularisation gamma.
 * Replaces a KernelType object's construction, e.g. Gaussian2DKernel(gamma, W, H)
 * (cpp/kernels.h:632-641), Gaussian3DKernel (:714-725),
 * LogSignArrayGaussian2DKernel (:1036-1045).  device < 0 selects the current device. */
int wdl_create(wdl_ctx** ctx, int device, int W, int H, int D, double gamma, int precision,
               int domain);
int wdl_destroy(wdl_ctx* ctx);
/* Waits for the context's stream. */
int wdl_synchronize(wdl_ctx* ctx);
/* Bytes of device memory a wdl_gradient_both / wdl_evaluate_both call with these
 * sizes allocates (iterate store + workspace). */
size_t wdl_eval_bytes(const wdl_ctx* ctx, int P, int K, int L);

/* ---- KernelType operator (host pointers) ---------------------------------
 * Gaussian2DKernel::convolve / convolveAdjoint (cpp/kernels.h:669-704),
 * Gaussian3DKernel::convolve (:762-811): out_v = G (*) u_v for nvectors stacked
 * images; the operator is symmetric, so the adjoint is the same call.  out may
 * alias u. */
int wdl_convolve(wdl_ctx* ctx, const double* u, double* out, int nvectors);
/* LogSignArrayGaussian2DKernel::log_convolve (cpp/kernels.h:1073-1115). */
int wdl_log_convolve(wdl_ctx* ctx, const double* log_u, double* out, int nvectors);
/* log_convolve_signArray (cpp/kernels.h:1117-1163): signs (bit=1 means >= 0,
 * bit i of byte i/8, cpp/signArray.h:8-22) are read for the input and
 * overwritten with the output's signs. */
int wdl_log_convolve_signed(wdl_ctx* ctx, const double* log_u, unsigned char* signs, double* out,
                            int nvectors);

/* ---- Hot path (host pointers) ------------------------------------------------
 * compute_gradient_both / compute_gradient_both_log_signArray
 * (cpp/inverseWasserstein.h:544-674, :678-814) for P histograms in one call:
 * the device-resident replacement of the per-histogram loop of evaluate_both
 * (:1052-1113).  atoms [K*N] and weights [P*K] are normalised first
 * (Problem::normalize_values, :53-74).
 *   result_la   [P*K]  raw weight gradient of each histogram (resultLa)
 *   result_dic  [K*N]  raw dictionary gradient summed over the P histograms, or
 *                      NULL when only the weight gradient is wanted (weights
 *                      fitted onto a fixed dictionary): the kernel-domain forms
 *                      then skip the dictionary recursion, a third of the work
 *   bary        [P*N]  barycenters, or NULL
 *   loss        [P]    loss of each barycenter against its observation, or NULL
 *   b_init      [P*K*N] initial scalings b[0] (warm restart), or NULL for ones
 *   b_last      [P*K*N] receives b[L] (warm restart store), or NULL */
int wdl_gradient_both(wdl_ctx* ctx, int P, int K, int L, int loss_type, const double* atoms,
                      const double* weights, const double* observed, const double* b_init,
                      double* result_la, double* result_dic, double* bary, double* loss,
                      double* b_last);

/* evaluate_both (cpp/inverseWasserstein.h:986-1145) with exp_weight = true:
 * x[n] -> objective *f and gradient g[n], n = P*K + K*N.  b_storage / b_last as
 * above (warm restart, :1057-1061, :1081-1085); bary [P*N] or NULL. */
int wdl_evaluate_both(wdl_ctx* ctx, int P, int K, int L, int loss_type, double scale_dic,
                      const double* x, double* g, int n, const double* observed, double* f,
                      const double* b_storage, double* b_last, double* bary);

/* WassersteinRegression::regress_both (cpp/inverseWasserstein.h:362-423) with
 * liblbfgs' algorithm on the device (cpp/lbfgs/lbfgs.c:256-654, strong-Wolfe
 * backtracking :772-867, m = 6, ftol 1e-4, wolfe 0.9, 20 trials per line
 * search, the reference's epsilon argument 1e-50 makes it run max_iterations):
 * solution [n = P*K + K*N] holds the weights and atoms in the original domain
 * on entry and the optimised, normalised ones on exit (the reference's
 * transform to [scaled log-weights, log-atoms] and back, :389-401, :424-448).
 * Every objective evaluation is this context's evaluate_both; the optimisation
 * vectors (x, gradient, previous point, direction, the 6 correction pairs) stay
 * on the device and the host reads one status word per evaluation.
 * warm_restart != 0: runs of 10 iterations, b[L] of each run kept on the device
 * as the next run's b[0] (:368-384, :407-416; max_iterations >= 10).
 * status = liblbfgs' return code of the last run, *f its final objective,
 * *evaluations the objective evaluations (any of the three may be NULL). */
int wdl_regress_both(wdl_ctx* ctx, int P, int K, int L, int loss_type, double scale_dic, double* solution,
                     const double* observed, int max_iterations, double epsilon, int warm_restart,
                     int* status, double* f, int* evaluations);

/* WassersteinBarycenter::compute_barycenter / _log (cpp/inverseWasserstein.h:115-201):
 * forward Bregman projections only, for P weight vectors against one set of atoms.
 * bary [P*N]. */
int wdl_barycenter(wdl_ctx* ctx, int P, int K, int L, const double* atoms, const double* weights,
                   double* bary);

/* ---- Batched independent problems ----------------------------------------------
 * Many independent problems in ONE persistent launch: each its own grid (2-D,
 * sides up to the context's, which must be a WDL_TF32 / WDL_SPLIT_BF16 kernel-
 * domain context of sides <= 128), atom count, iteration count, histogram count
 * and mode; all share the context's gamma.  Per problem, with host pointers:
 *   WDL_MODE_WEIGHTS     forward + weight recursion: result_la [P*K] (raw
 *                        resultLa), loss [P]; the dictionary recursion is skipped
 *                        (weight fitting / projection onto fixed atoms)
 *   WDL_MODE_BOTH        compute_gradient_both: result_la, result_dic [K*N]
 *                        (summed over P), loss
 *   WDL_MODE_BARYCENTER  forward only: bary [P*N] (compute_barycenter)
 * Any output pointer may be NULL.  No reference counterpart (the reference runs
 * one problem at a time); each problem's results equal a separate
 * wdl_gradient_both / wdl_barycenter call on its own grid. */
enum { WDL_MODE_WEIGHTS = 0, WDL_MODE_BOTH = 1, WDL_MODE_BARYCENTER = 2 };
typedef struct {
  int W, H, K, L, P, loss_type, mode;
  const double* atoms;     /* [K*N] */
  const double* weights;   /* [P*K] */
  const double* observed;  /* [P*N], unused for WDL_MODE_BARYCENTER */
  double* result_la;       /* [P*K] or NULL */
  double* result_dic;      /* [K*N] or NULL (WDL_MODE_BOTH) */
  double* bary;            /* [P*N] or NULL */
  double* loss;            /* [P] or NULL */
} wdl_problem;
int wdl_batch_run(wdl_ctx* ctx, const wdl_problem* problems, int nproblems);

/* ---- Batched weight fitting, L-BFGS on the device --------------------------------
 * Fits the barycentric weights of every histogram of every problem onto the
 * problem's fixed atoms: one L-BFGS per histogram over x in R^K with weights =
 * softmax(x) (the reference's log-domain weights with scaleDictionary 1,
 * cpp/inverseWasserstein.h:1000-1020, :1124-1133), liblbfgs' algorithm and
 * constants as regress_both sets them (m = 6, strong-Wolfe backtracking, ftol
 * 1e-4, wolfe 0.9, 20 trials; cpp/inverseWasserstein.h:362-372,
 * cpp/lbfgs/lbfgs.c:256-654, :772-867), max_iterations accepted steps, stop
 * when |g| / max(1, |x|) <= epsilon.  Every round evaluates all active
 * histograms in one launch of the fused kernel (wdl_batch_run's layout) and
 * advances every optimisation on the device; the round is a CUDA graph.
 * Context as for wdl_batch_run.  status[p] is liblbfgs' return code, or
 * WDL_FIT_OVERFLOW when the kernel-domain evaluation at the returned weights is
 * not finite (scalings beyond the float range: run that histogram in the log
 * domain).  loss[p] is the loss at the returned weights.  The reference's
 * counterpart is regress_both with the atoms held fixed, one problem at a time
 * on the host. */
enum { WDL_FIT_OVERFLOW = -2000 };
typedef struct {
  int W, H, K, L, P, loss_type;
  const double* atoms;     /* [K*N] fixed dictionary */
  const double* observed;  /* [P*N] histograms to fit */
  const double* x0;        /* [P*K] starting log-weights, or NULL (uniform weights) */
  double* weights;         /* [P*K] out: fitted weights */
  double* loss;            /* [P] out */
  int* status;             /* [P] out */
  int* evaluations;        /* [P] out: objective evaluations used */
} wdl_fit_problem;
int wdl_fit_weights(wdl_ctx* ctx, const wdl_fit_problem* problems, int nproblems, int max_iterations,
                    double epsilon);
/* The same fits (same transform, algorithm, constants and status codes) for
 * P histograms on the context's own grid with the context's own evaluation:
 * any dimension (2-D or 3-D), precision and domain the context computes,
 * except the fused tensor-core form (use wdl_fit_weights there).  Every round
 * is one weights-only compute_gradient_both over the P histograms followed by
 * one step of every optimisation on the device; the rounds after the first
 * are one CUDA graph, and the host reads the done flags every few rounds.
 * Histograms that finished are evaluated along at their last point without
 * moving.  Host buffers: atoms [K*N], observed [P*N], x0 [P*K] or NULL;
 * outputs weights [P*K], loss [P], status [P], evaluations [P].  A non-finite
 * evaluation ends that fit with WDL_ERR_NONFINITE.  The reference's
 * counterpart is regress_both with the atoms held fixed, one histogram at a
 * time on the host. */
int wdl_fit_weights_operator(wdl_ctx* ctx, int P, int K, int L, int loss_type, const double* atoms,
                             const double* observed, const double* x0, int max_iterations, double epsilon,
                             double* weights, double* loss, int* status, int* evaluations);
/* The same fit in the LOG domain (compute_gradient_both_log_signArray,
 * cpp/inverseWasserstein.h:678-814, restricted to the forward pass, the loss
 * and the weight recursion), for problems whose kernel-domain scalings leave
 * the float range: ONE persistent launch in which every histogram's whole
 * L-BFGS fit runs on the device (one CTA per histogram up to sides of 32, a
 * cluster of 2, 4 or 16 CTAs up to 64, 128, 512; 8 where the GPU cannot
 * place 16-CTA clusters).  Context: 2-D,
 * WDL_DOMAIN_LOG, FP32 arithmetic;
 * its gamma serves every problem.  Sides <= 512, K <= 16, loss 1, 2 or 4.
 * status[p] is liblbfgs' return code, or WDL_ERR_NONFINITE if an evaluation
 * was not finite.  No reference counterpart beyond regress_both run one
 * problem at a time. */
int wdl_fit_weights_log(wdl_ctx* ctx, const wdl_fit_problem* problems, int nproblems, int max_iterations,
                        double epsilon);

/* ---- Device-resident forms (device pointers, stream as void*) ----------------
 * Same semantics as the host forms; no host<->device copies, no synchronisation.
 * f is a device double. */
int wdl_evaluate_both_device(wdl_ctx* ctx, int P, int K, int L, int loss_type, double scale_dic,
                             const double* x, double* g, int n, const double* observed, double* f,
                             const double* b_storage, double* b_last, double* bary, void* stream);
int wdl_gradient_both_device(wdl_ctx* ctx, int P, int K, int L, int loss_type, const double* atoms,
                             const double* weights, const double* observed, const double* b_init,
                             double* result_la, double* result_dic, double* bary, double* loss,
                             double* b_last, void* stream);
int wdl_convolve_device(wdl_ctx* ctx, const double* u, double* out, int nvectors, void* stream);
/* wdl_regress_both with solution and observed in device memory. */
int wdl_regress_both_device(wdl_ctx* ctx, int P, int K, int L, int loss_type, double scale_dic,
                            double* solution, const double* observed, int max_iterations, double epsilon,
                            int warm_restart, int* status, double* f, int* evaluations, void* stream);

/* No counterpart in the reference (which has no device code).  The operator of
 * wdl_convolve_device for callers that cannot allocate device memory while they
 * run (hosts that reserve all memory at start-up, processes under a device
 * memory cap or pool): it calls no cudaMalloc, cudaFree or other allocating
 * routine, and takes its scratch from one fixed 32 MiB device array inside the
 * library.  wdl_create reserves that array on the context's device (it looks
 * up the array's address, which loads the library's module there); the device
 * holds it until the process exits.  The caller passes device input and
 * output.  3 * nvectors * N * (4 bytes, or 8 for WDL_FP64) rounded up must fit
 * in the 32 MiB, otherwise WDL_ERR_INVALID_ARG (the message gives the limit).
 * All calls share the array: calls that overlap on the GPU race, so serialise
 * them.  On a tensor-core context with sides above 128 the first call for a
 * given image count may time the axis pass's tile variants, which synchronises
 * the stream; wdl_set_autotune(ctx, 0) beforehand keeps the default variant.
 * CUDA loads each kernel's code on its first launch in the process (lazy
 * loading); a caller that must see no driver allocation at all runs with
 * CUDA_MODULE_LOADING=EAGER or makes one call before its no-allocation phase. */
int wdl_convolve_device_noalloc(wdl_ctx* ctx, const double* u, double* out, int nvectors,
                                void* stream);

/* ---- Instrumentation ------------------------------------------------------------
 * Kernel launches issued by this context since creation (every kernel of this
 * library counts one), and the time in the dominant kernel (the separable
 * operator, or the fused Sinkhorn kernel on the tensor-core path) measured with
 * CUDA events on the launching stream since profiling was switched on
 * (level >= 1; the events synchronise each launch); conv_images counts the
 * separable-operator applications those launches performed (an image through
 * both axes is one).  Level 2 also records a
 * device-side phase trace of the fused kernel: wdl_phase_trace returns 27
 * values, for item types forward / dictionary / weights, 8 accumulated phase
 * times in ns (claim, dependency wait, prologue, first operator, mid step,
 * second operator, epilogue, completion) and the item count.  (The reference
 * only times whole L-BFGS iterations, cpp/chrono.h:52-78.) */
long long wdl_launch_count(const wdl_ctx* ctx);
int wdl_set_profiling(wdl_ctx* ctx, int level);
int wdl_phase_trace(wdl_ctx* ctx, double* out27);
int wdl_conv_profile(const wdl_ctx* ctx, double* conv_ms, long long* conv_launches,
                     double* conv_images);
/* Launch shapes the autotuner chose on this context: entry i has key {kind,
 * rows, row length, images, element bytes, signed} (kind 1 = log-domain axis
 * pass: variant = rows per block; kind 2 = tensor-core axis pass: variant =
 * output tile height, element bytes 2 for split BF16 and 4 for TF32), the
 * chosen variant and its time in ms.  wdl_autotune_count returns the number of
 * entries.  wdl_set_autotune(ctx, 0) stops this context from timing variants
 * on first calls (a latency-bound caller such as a request loop, where every
 * timing would also synchronise the stream); untuned shapes then take the
 * default variant.  On by default; WDL_AUTOTUNE=0 turns it off process-wide. */
int wdl_set_autotune(wdl_ctx* ctx, int on);
int wdl_autotune_count(const wdl_ctx* ctx);
int wdl_autotune_entry(const wdl_ctx* ctx, int i, long long* key6, int* choice, float* ms);
/* Failure detection of the fused tensor-core kernel (no reference counterpart;
 * the reference's only failure signal is a NaN loss that cancels L-BFGS,
 * cpp/inverseWasserstein.h:1180-1184).  Every wait of that kernel on another
 * work item is bounded; when a bound runs out the kernel's remaining items stop,
 * the kernel exits normally and the call returns WDL_ERR_TIMEOUT, with the
 * context still usable.  wdl_set_wait_limit sets the bound on one dependency
 * wait, in seconds (0 restores the default of 4 s; at most 60).
 * wdl_inject_fault(ctx, WDL_FAULT_DROP_FIRST_ITERATION) makes the host leave
 * the first forward iteration's items out of the next wdl_batch_run's work
 * table, so that the others wait on flags nothing publishes (one call only;
 * kind 0 cancels): a fault made on the host for testing that path. */
enum { WDL_FAULT_DROP_FIRST_ITERATION = 1 };
int wdl_set_wait_limit(wdl_ctx* ctx, double seconds);
int wdl_inject_fault(wdl_ctx* ctx, int kind);
/* Exponentials the log-domain operator evaluated while profiling (the
 * reference evaluates one per tap, N*(W+H) per image; taps whose terms are
 * below the sum's rounding are skipped here). */
int wdl_exp_profile(const wdl_ctx* ctx, double* executed_exps);

#ifdef __cplusplus
}
#endif
#endif /* WDL_H */
