// wdl_fit_weights_log: batched weight fitting in the LOG domain, one
// persistent launch for all problems, each problem's whole fit on the device.
//
// The log-domain evaluation is the reference's compute_gradient_both_log_signArray
// (cpp/inverseWasserstein.h:678-814) restricted to what weight fitting needs:
// the forward Bregman iterations with the tape (:700-720), the loss and its
// gradient (cpp/loss.h:19-90) and the weight recursion of the reverse pass
// (:730-812: the signed log-sum-exp operator, cpp/kernels.h:1117-1159), whose
// per-step dot products are resultLa.  Around it runs liblbfgs' algorithm
// (lbfgs_dev.cuh), as regress_both runs it around evaluate_both.
//
// Each problem gets a group of CTAs by its size: 1 (sides <= 32), a cluster of
// 2 (<= 64), 4 (<= 128) or 16 (above); a cluster splits every pass's rows and
// every elementwise loop and meets at cluster barriers.  The four classes run
// as four launches on their own streams, concurrently.  A group never waits
// on another group, so the launch needs no residency guarantee and has no
// spin-waits.  The separable log-sum-exp passes follow the CUDA-core
// operator's (conv_simt.cu): outward taps with the provably negligible tail
// cut, base-2 FP32, an odd SMEM row stride.
//
// Why: the uneven workload's problems (sides 32-192, K 3-8, L 25-100) each
// need ~1000 small launches per evaluation on the operator path, and their
// kernel-domain scalings leave the float range, so they are log-domain fits.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "lbfgs_dev.cuh"
#include "log_group.cuh"
#include "wdl_internal.cuh"

namespace wdl {
namespace {

using namespace lbdev;

constexpr int kLfThreads = 256;
// CTAs per problem and rows per pass block, by size class; the largest class
// uses 16-CTA clusters (a non-portable size, falling back to 8) with 8-row
// blocks, so that a 192-row pass still gives every CTA rows.
constexpr int kGroups[4] = {1, 2, 4, 16};
inline int size_class(int W, int H) {
  const int m = W > H ? W : H;
  return m <= 32 ? 0 : m <= 64 ? 1 : m <= 128 ? 2 : 3;
}
constexpr int kLfMaxK = 16;
constexpr float kLog2e = 1.4426950408889634f;
constexpr float kFloorF = -3.402823466e38f;

struct LogFitProblem {
  int W, H, K, L, loss_type;
  const float* latoms;   // [K][N] log of the normalised atoms
  const double* obs;     // [N]
  float *tb, *tcb, *tphi;  // tapes (log values): b [L+1][K][N], conv_b [L][K][N], phi [L][K][N]
  float *t1, *a;         // [N]: transposed intermediate, second operand / result
  float *u, *r;          // [K][N]
  float *gw, *blog;      // [N]
  uint8_t *sw, *ts;      // [K][N] signs, [N] intermediate signs
  double* part;          // [group][K + 1] partial sums (dot products, loss)
  double* v;             // L-BFGS vectors (pool_doubles(K))
  double* w64;           // [K] weights of the current trial point
  float* w32;
  LbState* st;
  int* flag;             // 1 while the fit needs another evaluation
};

__device__ __forceinline__ void cluster_barrier() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

template <int G>
__device__ __forceinline__ void group_sync() {
  __syncthreads();
  if (G > 1) cluster_barrier();
}

__device__ double block_sum_d(double v, double* sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) sh[w] = v;
  __syncthreads();
  double t = 0;
  for (int i = 0; i < kLfThreads / 32; ++i) t += sh[i];
  __syncthreads();
  return t;  // in every thread
}

// One separable log-sum-exp axis pass of one image ([R][C] -> [C][R]), the
// rows shared among the group: out[c][r] = log sum_k s_k exp(-(c-k)^2/gamma +
// in[r][k]) (signs optional, in and out sign arrays distinct), as the
// CUDA-core operator's pass: rows staged with a halo, four neighbouring outputs
// of a row per thread in one running-maximum pass (log_group.cuh).
template <bool SIGNED, int G, int LR>
__device__ void lse_pass(const float* __restrict__ in, float* __restrict__ out, int R, int C, float gamma,
                         const uint8_t* __restrict__ in_sign, uint8_t* __restrict__ out_sign, float* sm,
                         int rank) {
  using namespace lse;
  const int CP = log_cp(C), SP = log_sp(C);
  float* rows = sm;
  float* lk = rows + LR * CP;
  float* xmax = lk + C;
  uint8_t* sg = reinterpret_cast<uint8_t*>(xmax + LR);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int G4 = (C + 3) >> 2;
  const bool full = (C & 3) == 0;
  __syncthreads();
  for (int d = tid; d < C; d += kLfThreads) lk[d] = -float(d) * float(d) / gamma * kLog2e;
  for (int rb = rank; rb * LR < R; rb += G) {
    const int r0 = rb * LR, nr = min(LR, R - r0);
    __syncthreads();
    for (int rr = warp; rr < LR; rr += kLfThreads / 32) {
      float* rw = rows + rr * CP + kHalo;
      uint8_t* sw = sg + rr * SP + kHalo;
      for (int k = lane; k < kHalo; k += 32) {
        rw[-kHalo + k] = LogOps<float>::kNone;
        rw[C + k] = LogOps<float>::kNone;
        if (SIGNED) {
          sw[-kHalo + k] = 1;
          sw[C + k] = 1;
        }
      }
      float vm = kFloorF;
      for (int k = lane; k < C; k += 32) {
        float v = kFloorF;
        uint8_t sv = 1;
        if (rr < nr) {
          v = in[(size_t)(r0 + rr) * C + k] * kLog2e;
          if (SIGNED) sv = in_sign[(size_t)(r0 + rr) * C + k];
        }
        rw[k] = v;
        if (SIGNED) sw[k] = sv;
        vm = fmaxf(vm, v);
      }
      for (int o = 16; o > 0; o >>= 1) vm = fmaxf(vm, __shfl_xor_sync(0xffffffffu, vm, o));
      if (lane == 0) xmax[rr] = vm;
    }
    __syncthreads();
    for (int e = tid; e < LR * G4; e += kLfThreads) {
      const int gi = e / LR, rr = e - gi * LR;
      if (rr >= nr) continue;
      const int c0 = 4 * gi;
      const float* row = rows + rr * CP + kHalo;
      const uint8_t* sgn = sg + rr * SP + kHalo;
      float v[4];
      bool pos[4];
      if (full) log_group<float, SIGNED, true>(row, sgn, lk, xmax[rr], c0, C, v, pos);
      else log_group<float, SIGNED, false>(row, sgn, lk, xmax[rr], c0, C, v, pos);
      const int nv = min(4, C - c0);
      for (int j = 0; j < nv; ++j) {
        const size_t o = (size_t)(c0 + j) * R + (r0 + rr);
        out[o] = v[j];
        if (SIGNED) out_sign[o] = pos[j] ? 1 : 0;
      }
    }
  }
}

// The 2-D operator: x pass into t1 (transposed), y pass into out.
template <bool SIGNED, int G, int LR>
__device__ void lse_image(const float* in, float* out, const LogFitProblem& p, float gamma, uint8_t* signs,
                          float* sm, int rank) {
  lse_pass<SIGNED, G, LR>(in, p.t1, p.H, p.W, gamma, signs, p.ts, sm, rank);
  group_sync<G>();
  lse_pass<SIGNED, G, LR>(p.t1, out, p.W, p.H, gamma, p.ts, signs, sm, rank);
  group_sync<G>();
}

template <int G, int LR>
__global__ void __launch_bounds__(kLfThreads)
    log_fit_kernel(const LogFitProblem* __restrict__ probs, int nprob, LbParam prm, float gamma, int max_evals) {
  extern __shared__ float sm[];
  __shared__ double sh[kLfThreads / 32];
  __shared__ double s_la[kLfMaxK + 1];
  __shared__ float s_lam[kLfMaxK];
  __shared__ int s_flag;
  const int q = blockIdx.x / G, rank = blockIdx.x - q * G;
  if (q >= nprob) return;
  const LogFitProblem p = probs[q];
  const int K = p.K, L = p.L, tid = threadIdx.x;
  const size_t N = (size_t)p.W * p.H, KN = (size_t)K * N;
  const size_t gstride = (size_t)G * kLfThreads, g0 = (size_t)rank * kLfThreads + tid;

  for (int e = 0; e < max_evals; ++e) {
    group_sync<G>();
    if (tid == 0) s_flag = *(volatile const int*)p.flag;
    if (tid < K) s_lam[tid] = *(volatile const float*)(p.w32 + tid);
    __syncthreads();
    if (!s_flag) break;

    // ---- forward (:700-720): b0 = 0 (log of ones) --------------------------------
    for (size_t i = g0; i < KN; i += gstride) p.tb[i] = 0.f;
    group_sync<G>();
    for (int it = 1; it <= L; ++it) {
      const float* bprev = p.tb + (size_t)(it - 1) * KN;
      float* cb = p.tcb + (size_t)(it - 1) * KN;
      float* ph = p.tphi + (size_t)(it - 1) * KN;
      for (int k = 0; k < K; ++k) {
        lse_image<false, G, LR>(bprev + k * N, cb + k * N, p, gamma, nullptr, sm, rank);
        for (size_t j = g0; j < N; j += gstride) p.a[j] = p.latoms[k * N + j] - cb[k * N + j];
        group_sync<G>();
        lse_image<false, G, LR>(p.a, ph + k * N, p, gamma, nullptr, sm, rank);
      }
      float* bnext = p.tb + (size_t)it * KN;
      for (size_t j = g0; j < N; j += gstride) {
        float s = 0.f;
        for (int k = 0; k < K; ++k) s += ph[k * N + j] * s_lam[k];
        p.blog[j] = s;
        for (int k = 0; k < K; ++k) bnext[k * N + j] = s - ph[k * N + j];
      }
      group_sync<G>();
    }
    // ---- loss and its gradient (cpp/loss.h:19-90); gw = g * bary (:633-635) --------
    double lacc = 0;
    for (size_t j = g0; j < N; j += gstride) {
      const float v1 = expf(p.blog[j]);
      const double o = p.obs[j];
      const float v2 = (float)o;
      float g;
      if (p.loss_type == WDL_LOSS_TV) {
        lacc += fabs((double)v1 - o);
        g = v1 - v2 > 0.f ? 0.5f : -0.5f;
      } else if (p.loss_type == WDL_LOSS_QUADRATIC) {
        const double d = (double)v1 - o;
        lacc += d * d;
        g = 2.f * (v1 - v2);
      } else {
        const double rr = (double)v1 / o;
        lacc += (double)v1 * log(rr > kEpsilon ? rr : kEpsilon) - (double)v1 + o;
        const float q2 = v1 / v2;
        g = q2 > 0.f ? logf(q2) : (float)kLogEpsilon;
      }
      p.gw[j] = g * v1;
    }
    lacc = block_sum_d(lacc, sh);
    if (tid == 0) p.part[rank * (K + 1) + K] = lacc;
    // ---- reverse pass, weight recursion (:730-812) -------------------------------------
    for (size_t i = g0; i < KN; i += gstride) p.r[i] = 0.f;
    double dacc[kLfMaxK];
    for (int k = 0; k < K; ++k) dacc[k] = 0;
    group_sync<G>();
    for (int s = L; s >= 1; --s) {
      const float* phs = p.tphi + (size_t)(s - 1) * KN;
      for (int k = 0; k < K; ++k) {
        const float l = s_lam[k];
        double acc = 0;
        for (size_t j = g0; j < N; j += gstride) {
          const size_t i = k * N + j;
          const float ph = phs[i], g = p.gw[j];
          acc += (double)ph * (double)g;
          const float y = l * g + p.r[i];
          p.sw[i] = y >= 0.f;
          p.u[i] = logf(fabsf(y)) - ph;
        }
        dacc[k] += acc;
      }
      group_sync<G>();
      if (s == 1) break;
      const float* cbs = p.tcb + (size_t)(s - 1) * KN;
      const float* bp = p.tb + (size_t)(s - 1) * KN;
      for (int k = 0; k < K; ++k) {
        lse_image<true, G, LR>(p.u + k * N, p.a, p, gamma, p.sw + k * N, sm, rank);
        for (size_t j = g0; j < N; j += gstride)
          p.u[k * N + j] = p.a[j] + (p.latoms[k * N + j] - 2.f * cbs[k * N + j]);
        group_sync<G>();
        lse_image<true, G, LR>(p.u + k * N, p.a, p, gamma, p.sw + k * N, sm, rank);
        for (size_t j = g0; j < N; j += gstride) {
          const float ex = expf(p.a[j] + bp[k * N + j]);
          p.r[k * N + j] = p.sw[k * N + j] ? ex : -ex;
        }
        group_sync<G>();
      }
      for (size_t j = g0; j < N; j += gstride) {
        float sg = 0.f;
        for (int k = 0; k < K; ++k) sg -= p.r[k * N + j];
        p.gw[j] = sg;
      }
      group_sync<G>();
    }
    for (int k = 0; k < K; ++k) {
      const double t = block_sum_d(dacc[k], sh);
      if (tid == 0) p.part[rank * (K + 1) + k] = t;
    }
    group_sync<G>();
    // ---- one L-BFGS step (rank 0, thread 0) -----------------------------------------
    if (rank == 0 && tid == 0) {
      for (int k = 0; k <= K; ++k) {
        double t = 0;
        for (int g = 0; g < G; ++g) t += p.part[g * (K + 1) + k];
        s_la[k] = t;
      }
      const double f = p.loss_type == WDL_LOSS_TV ? 0.5 * s_la[K] : s_la[K];
      LbState st = *p.st;
      lbfgs_advance(st, p.v, f, s_la, p.w64, p.w32, prm, WDL_ERR_NONFINITE);
      *p.st = st;
      *p.flag = st.phase == 2 ? 0 : 1;
      __threadfence();
    }
  }
}

inline size_t a256(size_t b) { return (b + 255) & ~size_t(255); }

size_t lse_smem(int C, int LR) {
  return ((size_t)LR * lse::log_cp(C) + C + LR) * sizeof(float) + (size_t)LR * lse::log_sp(C) + 16;
}

template <int G, int LR>
int launch_log_fit(wdl_ctx* ctx, const LogFitProblem* d_probs, int n, const LbParam& prm, int max_evals,
                   int maxC, cudaStream_t s) {
  const size_t smem = lse_smem(maxC, LR);
  auto kern = log_fit_kernel<G, LR>;
  if (smem > 48 * 1024)
    WDL_CUDA_TRY(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  if (G > 8)
    WDL_CUDA_TRY(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
  if (G == 1) {
    kern<<<n, kLfThreads, smem, s>>>(d_probs, n, prm, (float)ctx->gamma, max_evals);
  } else {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(n * G));
    cfg.blockDim = dim3(kLfThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = G;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    WDL_CUDA_TRY(ctx, cudaLaunchKernelEx(&cfg, kern, d_probs, n, prm, (float)ctx->gamma, max_evals));
  }
  WDL_LAUNCH_CHECK(ctx);
  return WDL_OK;
}

// Whether a 16-CTA cluster of this kernel can be resident at all (a
// non-portable size; otherwise the class runs on 8-CTA clusters).
bool big_clusters_fit(size_t smem) {
  auto kern = log_fit_kernel<16, 8>;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess ||
      (smem > 48 * 1024 &&
       cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)) {
    cudaGetLastError();
    return false;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(16);
  cfg.blockDim = dim3(kLfThreads);
  cfg.dynamicSmemBytes = smem;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = 16;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int nclusters = 0;
  const cudaError_t e = cudaOccupancyMaxActiveClusters(&nclusters, kern, &cfg);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return nclusters > 0;
}

}  // namespace
}  // namespace wdl

using namespace wdl;

extern "C" int wdl_fit_weights_log(wdl_ctx* ctx, const wdl_fit_problem* fp, int nprob, int max_iterations,
                                   double epsilon) {
  if (!ctx) return WDL_ERR_INVALID_ARG;
  if (!fp || nprob < 1 || max_iterations < 0 || !(epsilon >= 0))
    return set_error(ctx, WDL_ERR_INVALID_ARG, "bad arguments");
  if (ctx->domain != WDL_DOMAIN_LOG || ctx->ndim != 2 || ctx->precision == WDL_FP64)
    return set_error(ctx, WDL_ERR_UNSUPPORTED, "wdl_fit_weights_log needs a 2-D log-domain FP32 context");
  if (cudaSetDevice(ctx->device) != cudaSuccess) return set_error(ctx, WDL_ERR_CUDA, "cudaSetDevice failed");
  cudaStream_t s = ctx->stream;
  // One entry per histogram; the two size classes get their own launches.
  struct Entry {
    int q, p, cls;
    size_t off, bytes;
  };
  std::vector<Entry> ent;
  for (int q = 0; q < nprob; ++q) {
    const wdl_fit_problem& f = fp[q];
    if (f.W < 1 || f.H < 1 || f.W > 512 || f.H > 512 || f.K < 1 || f.K > kLfMaxK || f.L < 1 || f.P < 1 ||
        !f.atoms || !f.observed || !f.weights || !f.loss || !f.status || !f.evaluations ||
        f.loss_type < WDL_LOSS_TV || f.loss_type > WDL_LOSS_KL || f.loss_type == WDL_LOSS_WASSERSTEIN)
      return set_error(ctx, WDL_ERR_INVALID_ARG,
                       "fit problem " + std::to_string(q) + ": bad sizes, pointers or loss (sides <= 512, K <= 16)");
    for (int p = 0; p < f.P; ++p) ent.push_back({q, p, size_class(f.W, f.H), 0, 0});
  }
  // per-entry device footprint
  auto footprint = [&](const wdl_fit_problem& f, int G) {
    const size_t N = (size_t)f.W * f.H, K = f.K, L = f.L, KN = K * N;
    size_t b = 0;
    b += a256(KN * 4);                  // latoms
    b += a256(N * 8);                   // obs
    b += a256((L + 1) * KN * 4) + 2 * a256(L * KN * 4);  // tapes
    b += 4 * a256(N * 4) + 2 * a256(KN * 4);             // t1, a, gw, blog, u, r
    b += a256(KN) + a256(N);            // sw, ts
    b += a256((size_t)G * (K + 1) * 8) + a256(pool_doubles((int)K) * 8) + a256(K * 8) + a256(K * 4);
    b += a256(sizeof(LbState)) + a256(sizeof(int));
    return b;
  };
  size_t free_b = 0, total_b = 0;
  WDL_CUDA_TRY(ctx, cudaMemGetInfo(&free_b, &total_b));
  const size_t budget = (size_t)(0.6 * (double)(free_b + ctx->arena.bytes));
  LbParam prm{max_iterations, 20, epsilon, 1e-4, 0.9, 1e-20, 1e20};
  const int max_evals = (max_iterations > 0 ? max_iterations : 1000) * (prm.max_linesearch + 1) + 2;
  size_t done = 0;
  while (done < ent.size()) {
    // a wave: as many entries as fit the budget (at least one)
    size_t used = a256(sizeof(LogFitProblem) * ent.size()), end = done;
    while (end < ent.size()) {
      const wdl_fit_problem& f = fp[ent[end].q];
      const size_t b = footprint(f, kGroups[ent[end].cls]);
      if (end > done && used + b > budget) break;
      ent[end].off = used;
      ent[end].bytes = b;
      used += b;
      ++end;
    }
    int rc;
    if ((rc = ensure_arena(ctx, used))) return rc;
    char* base = static_cast<char*>(ctx->arena.ptr);
    // host-side inputs, descriptors and initial states
    std::vector<LogFitProblem> desc;
    int maxC[4] = {0, 0, 0, 0}, cnt[4] = {0, 0, 0, 0};
    std::vector<size_t> order;
    for (int cls = 0; cls < 4; ++cls) {
      const size_t first = order.size();
      for (size_t e = done; e < end; ++e)
        if (ent[e].cls == cls) order.push_back(e);
      // heaviest problems first (one operator pass costs ~N (W + H), K L of
      // them per evaluation): the CTAs are scheduled in launch order, so this
      // shortens the tail of the launch
      auto work = [&](size_t e) {
        const wdl_fit_problem& f = fp[ent[e].q];
        return (double)f.K * f.L * f.W * f.H * (f.W + f.H);
      };
      std::stable_sort(order.begin() + first, order.end(),
                       [&](size_t x, size_t y) { return work(x) > work(y); });
    }
    for (size_t e : order) {
      const Entry& en = ent[e];
      const wdl_fit_problem& f = fp[en.q];
      const int G = kGroups[en.cls];
      const size_t N = (size_t)f.W * f.H, K = f.K, L = f.L, KN = K * N;
      char* c = base + en.off;
      auto take = [&](size_t bytes) {
        char* r = c;
        c += a256(bytes);
        return r;
      };
      LogFitProblem d{};
      d.W = f.W;
      d.H = f.H;
      d.K = f.K;
      d.L = f.L;
      d.loss_type = f.loss_type;
      float* lat = reinterpret_cast<float*>(take(KN * 4));
      double* obs = reinterpret_cast<double*>(take(N * 8));
      d.latoms = lat;
      d.obs = obs;
      d.tb = reinterpret_cast<float*>(take((L + 1) * KN * 4));
      d.tcb = reinterpret_cast<float*>(take(L * KN * 4));
      d.tphi = reinterpret_cast<float*>(take(L * KN * 4));
      d.t1 = reinterpret_cast<float*>(take(N * 4));
      d.a = reinterpret_cast<float*>(take(N * 4));
      d.gw = reinterpret_cast<float*>(take(N * 4));
      d.blog = reinterpret_cast<float*>(take(N * 4));
      d.u = reinterpret_cast<float*>(take(KN * 4));
      d.r = reinterpret_cast<float*>(take(KN * 4));
      d.sw = reinterpret_cast<uint8_t*>(take(KN));
      d.ts = reinterpret_cast<uint8_t*>(take(N));
      d.part = reinterpret_cast<double*>(take((size_t)G * (K + 1) * 8));
      d.v = reinterpret_cast<double*>(take(pool_doubles((int)K) * 8));
      d.w64 = reinterpret_cast<double*>(take(K * 8));
      d.w32 = reinterpret_cast<float*>(take(K * 4));
      d.st = reinterpret_cast<LbState*>(take(sizeof(LbState)));
      d.flag = reinterpret_cast<int*>(take(sizeof(int)));
      // log of the normalised atoms (Problem::normalize_values, :53-74), FP64 then FP32
      std::vector<float> hl(KN);
      for (size_t k = 0; k < K; ++k) {
        double sum = 0;
        for (size_t j = 0; j < N; ++j) sum += f.atoms[k * N + j];
        for (size_t j = 0; j < N; ++j) hl[k * N + j] = (float)std::log(f.atoms[k * N + j] / sum);
      }
      std::vector<double> hv(pool_doubles((int)K), 0.0), hw(K);
      std::vector<float> hw32(K);
      for (size_t k = 0; k < K; ++k) hv[k] = f.x0 ? f.x0[(size_t)en.p * K + k] : 0.0;
      {
        double mx = hv[0];
        for (size_t k = 1; k < K; ++k) mx = hv[k] > mx ? hv[k] : mx;
        double ssum = 0;
        for (size_t k = 0; k < K; ++k) ssum += std::exp(hv[k] - mx);
        for (size_t k = 0; k < K; ++k) {
          hw[k] = std::exp(hv[k] - mx) / ssum;
          hw32[k] = (float)hw[k];
        }
      }
      LbState st{};
      st.K = (int)K;
      const int one = 1;
      WDL_CUDA_TRY(ctx, cudaMemcpyAsync(lat, hl.data(), KN * 4, cudaMemcpyHostToDevice, s));
      WDL_CUDA_TRY(ctx, cudaMemcpyAsync(obs, f.observed + (size_t)en.p * N, N * 8, cudaMemcpyHostToDevice, s));
      WDL_CUDA_TRY(ctx, cudaMemcpyAsync(d.v, hv.data(), hv.size() * 8, cudaMemcpyHostToDevice, s));
      WDL_CUDA_TRY(ctx, cudaMemcpyAsync(d.w64, hw.data(), K * 8, cudaMemcpyHostToDevice, s));
      WDL_CUDA_TRY(ctx, cudaMemcpyAsync(d.w32, hw32.data(), K * 4, cudaMemcpyHostToDevice, s));
      WDL_CUDA_TRY(ctx, cudaMemcpyAsync(d.st, &st, sizeof(st), cudaMemcpyHostToDevice, s));
      WDL_CUDA_TRY(ctx, cudaMemcpyAsync(d.flag, &one, sizeof(int), cudaMemcpyHostToDevice, s));
      WDL_CUDA_TRY(ctx, cudaStreamSynchronize(s));  // the host vectors above are locals
      desc.push_back(d);
      const int C = f.W > f.H ? f.W : f.H;
      if (C > maxC[en.cls]) maxC[en.cls] = C;
      cnt[en.cls]++;
    }
    LogFitProblem* d_probs = reinterpret_cast<LogFitProblem*>(base);
    WDL_CUDA_TRY(ctx, cudaMemcpyAsync(d_probs, desc.data(), desc.size() * sizeof(LogFitProblem),
                                      cudaMemcpyHostToDevice, s));
    {  // the four classes concurrently, each on a stream of its own
      cudaStream_t cs[4] = {nullptr, nullptr, nullptr, nullptr};
      int first = 0;
      rc = WDL_OK;
      for (int cls = 0; cls < 4 && rc == WDL_OK; ++cls) {
        if (!cnt[cls]) continue;
        cudaError_t e = cudaStreamCreateWithFlags(&cs[cls], cudaStreamNonBlocking);
        if (e != cudaSuccess) {
          rc = cuda_error(ctx, e, "cudaStreamCreateWithFlags");
          break;
        }
        const LogFitProblem* dp = d_probs + first;
        switch (cls) {
          case 0: rc = launch_log_fit<1, 16>(ctx, dp, cnt[0], prm, max_evals, maxC[0], cs[0]); break;
          case 1: rc = launch_log_fit<2, 16>(ctx, dp, cnt[1], prm, max_evals, maxC[1], cs[1]); break;
          case 2: rc = launch_log_fit<4, 16>(ctx, dp, cnt[2], prm, max_evals, maxC[2], cs[2]); break;
          default:
            if (big_clusters_fit(lse_smem(maxC[3], 8))) {
              rc = launch_log_fit<16, 8>(ctx, dp, cnt[3], prm, max_evals, maxC[3], cs[3]);
            } else {
              rc = launch_log_fit<8, 16>(ctx, dp, cnt[3], prm, max_evals, maxC[3], cs[3]);
            }
            break;
        }
        first += cnt[cls];
      }
      for (int cls = 0; cls < 4; ++cls) {
        if (!cs[cls]) continue;
        const cudaError_t e = cudaStreamSynchronize(cs[cls]);
        if (e != cudaSuccess && rc == WDL_OK) rc = cuda_error(ctx, e, "log-domain fit");
        cudaStreamDestroy(cs[cls]);
      }
      if (rc) return rc;
    }
    // results
    for (size_t i = 0; i < order.size(); ++i) {
      const Entry& en = ent[order[i]];
      const wdl_fit_problem& f = fp[en.q];
      const int K = f.K;
      LbState st{};
      std::vector<double> x(K);
      WDL_CUDA_TRY(ctx, cudaMemcpyAsync(&st, desc[i].st, sizeof(st), cudaMemcpyDeviceToHost, s));
      WDL_CUDA_TRY(ctx, cudaMemcpyAsync(x.data(), desc[i].v, K * 8, cudaMemcpyDeviceToHost, s));
      WDL_CUDA_TRY(ctx, cudaStreamSynchronize(s));
      double mx = x[0];
      for (int k = 1; k < K; ++k) mx = x[k] > mx ? x[k] : mx;
      double ssum = 0;
      for (int k = 0; k < K; ++k) ssum += std::exp(x[k] - mx);
      for (int k = 0; k < K; ++k) f.weights[(size_t)en.p * K + k] = std::exp(x[k] - mx) / ssum;
      f.loss[en.p] = st.phase == 2 ? st.fret : st.f;
      f.status[en.p] = st.phase == 2 ? st.status : kMaximumIteration;
      f.evaluations[en.p] = st.evals;
    }
    done = end;
  }
  return WDL_OK;
}
