// Device-resident Sinkhorn-barycenter forward pass, loss, and reverse pass
// through the stored iterates, for P histograms at once.
//
// This is the batched replacement of the per-histogram loop of evaluate_both
// (cpp/inverseWasserstein.h:1052-1113) around compute_gradient_both (:544-674)
// and compute_gradient_both_log_signArray (:678-814).  Histograms are laid out
// [P][K][N] (histogram, atom, pixel) so that one launch of the separable
// operator covers every histogram and atom of a step.  The dictionary and
// weight recursions of the reverse pass are independent of each other (the
// reference runs them one after the other); here they advance together, one
// step s per round, so each round's two operator applications cover 2*P*K images
// in one launch.  Elementwise work between operator applications is fused into
// one kernel per round; every reduction over the grid or the batch (loss,
// weight-gradient dot products, the sum of the dictionary gradient over P) runs
// in FP64.
#include <cmath>
#include <cstring>
#include <functional>

#include "wdl_internal.cuh"
#include "wdl_math.cuh"

namespace wdl {
namespace {

template <typename T>
__device__ __forceinline__ T d_exp(T x);
template <>
__device__ __forceinline__ float d_exp<float>(float x) { return expf(x); }
template <>
__device__ __forceinline__ double d_exp<double>(double x) { return exp(x); }
template <typename T>
__device__ __forceinline__ T d_log(T x);
template <>
__device__ __forceinline__ float d_log<float>(float x) { return logf(x); }
template <>
__device__ __forceinline__ double d_log<double>(double x) { return log(x); }
// Natural log of a magnitude feeding a log-domain operand: FP32 takes the
// hardware base-2 logarithm times ln 2 (absolute error ~2e-7, i.e. ~2e-7
// relative on the scaling it encodes; a log-domain value of magnitude >= 2 is
// rounded more coarsely than that anyway); FP64 the library log.
template <typename T>
__device__ __forceinline__ T d_log_mag(T x);
template <>
__device__ __forceinline__ float d_log_mag<float>(float x) {
  float y;
  asm("lg2.approx.f32 %0, %1;" : "=f"(y) : "f"(fabsf(x)));
  return y * 0.6931471805599453f;
}
template <>
__device__ __forceinline__ double d_log_mag<double>(double x) { return log(fabs(x)); }

// safe_log = log(max(EPSILON, x)) (cpp/loss.h:3-5).
template <typename T>
__device__ __forceinline__ T safe_log(T x);
template <>
__device__ __forceinline__ double safe_log<double>(double x) {
  return log(x > kEpsilon ? x : kEpsilon);
}
template <>
__device__ __forceinline__ float safe_log<float>(float x) {
  return x > 0.f ? logf(x) : float(kLogEpsilon);
}

// Logarithms that are summed in FP64 (grid reductions, the geometric mean over
// atoms): FP64 mode uses log directly; FP32 mode uses the split form of
// log_f32_precise so the FP64 sum is not limited by logf's absolute error.
template <typename T>
__device__ __forceinline__ double acc_log(T x);
template <>
__device__ __forceinline__ double acc_log<double>(double x) { return log(x); }
template <>
__device__ __forceinline__ double acc_log<float>(float x) {
  return x > 0.f ? log_f32_precise(x) : (double)logf(x);
}
template <typename T>
__device__ __forceinline__ double acc_safe_log(T x);
template <>
__device__ __forceinline__ double acc_safe_log<double>(double x) {
  return log(x > kEpsilon ? x : kEpsilon);
}
template <>
__device__ __forceinline__ double acc_safe_log<float>(float x) {
  return x > 0.f ? log_f32_precise(x) : kLogEpsilon;
}
template <typename T>
__device__ __forceinline__ T exp_from(double s);
template <>
__device__ __forceinline__ double exp_from<double>(double s) { return exp(s); }
template <>
__device__ __forceinline__ float exp_from<float>(double s) { return exp_to_f32(s); }

__device__ __forceinline__ double block_sum(double v, double* sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = blockDim.x >> 5;
  __syncthreads();
  if (l == 0) sh[w] = v;
  __syncthreads();
  double t = 0;
  if (threadIdx.x < 32) {
    t = threadIdx.x < nw ? sh[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
  }
  return t;  // valid in thread 0
}

#define GRID_STRIDE(i, n) \
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < (n); i += (size_t)gridDim.x * blockDim.x)

template <typename T>
__global__ void k_cast(const double* __restrict__ in, T* __restrict__ out, size_t n) {
  GRID_STRIDE(i, n) out[i] = (T)in[i];
}
template <typename T>
__global__ void k_cast_back(const T* __restrict__ in, double* __restrict__ out, size_t n) {
  GRID_STRIDE(i, n) out[i] = (double)in[i];
}
template <typename T>
__global__ void k_fill(T* __restrict__ p, T v, size_t n) {
  GRID_STRIDE(i, n) p[i] = v;
}
template <typename T>
__global__ void k_log_of(const double* __restrict__ in, T* __restrict__ out, size_t n) {
  GRID_STRIDE(i, n) out[i] = (T)log(in[i]);
}

// Problem::normalize_values (cpp/inverseWasserstein.h:53-74), one row per block.
// With exp_scale != 0 the row is first mapped through exp(v / exp_scale)
// (evaluate_both's return to the original domain, :997-1011).
__global__ void k_normalise_rows(const double* __restrict__ in, double* __restrict__ out,
                                 size_t len, double exp_scale) {
  __shared__ double sh[32];
  const double* r = in + (size_t)blockIdx.x * len;
  double* o = out + (size_t)blockIdx.x * len;
  double s = 0;
  for (size_t j = threadIdx.x; j < len; j += blockDim.x) {
    double v = exp_scale != 0.0 ? exp(r[j] / exp_scale) : r[j];
    o[j] = v;
    s += v;
  }
  s = block_sum(s, sh);
  if (threadIdx.x == 0) sh[0] = s;
  __syncthreads();
  s = sh[0];
  for (size_t j = threadIdx.x; j < len; j += blockDim.x) o[j] = o[j] / s;
}

// ---------------- kernel-domain forward (cpp/inverseWasserstein.h:565-593) -----------
// Out-of-range scalings: with a narrow kernel the kernel-domain scalings grow
// with the iterations (past 1e60 within 50 iterations at gamma = 2 px^2 for
// dictionaries with empty regions), beyond the FP32 range where the reference's
// FP64 still holds them.  In FP32 a scaling then saturates (inf, or a 0 that
// turns the next ratio into inf or NaN), and later iterations can carry on with
// finite but meaningless values.  The FP32 forms record per histogram whether
// a scaling a or b was ever non-finite (range[p], when given), and such a
// histogram's barycenter is replaced by NaN after the forward pass, so its
// loss and gradients report the overflow as NaN, as the FP64 path would
// report one of its own.

// a = p / conv_b, the atoms shared by every histogram.
template <typename T>
__global__ void k_div_atoms(const T* __restrict__ atoms, const T* __restrict__ cb,
                            T* __restrict__ a, size_t KN, size_t total, int* __restrict__ range) {
  GRID_STRIDE(i, total) {
    const T v = atoms[i % KN] / cb[i];
    a[i] = v;
    if (range && !isfinite(v)) range[i / KN] = 1;
  }
}

// Weighted geometric mean over the K atoms and the next scalings b = bary / phi.
template <typename T>
__global__ void k_bary_b(const T* __restrict__ phi, const double* __restrict__ lam,
                         T* __restrict__ b, T* __restrict__ bary, int K, size_t N, size_t PN,
                         int* __restrict__ range) {
  GRID_STRIDE(idx, PN) {
    const size_t p = idx / N, j = idx - p * N;
    const T* ph = phi + p * K * N + j;
    double s = 0;
    for (int k = 0; k < K; ++k) s += acc_safe_log<T>(ph[k * N]) * lam[p * K + k];
    const T by = exp_from<T>(s);
    bary[idx] = by;
    if (b) {
      bool bad = false;
      for (int k = 0; k < K; ++k) {
        const T bv = by / ph[k * N];
        b[p * K * N + k * N + j] = bv;
        bad |= !isfinite(bv);
      }
      if (range && bad) range[p] = 1;
    }
  }
}

// NaN barycenters for the histograms whose scalings left the range.
template <typename T>
__global__ void k_poison_out_of_range(T* __restrict__ bary, const int* __restrict__ range, size_t N,
                                      size_t PN) {
  GRID_STRIDE(idx, PN) if (range[idx / N]) bary[idx] = T(NAN);
}

// ---------------- log-domain forward (:700-720, :167-196) ---------------------------
template <typename T>
__global__ void k_log_bary_b(const T* __restrict__ phi, const T* __restrict__ lam,
                             T* __restrict__ b, T* __restrict__ bary_log, int K, size_t N,
                             size_t PN) {
  GRID_STRIDE(idx, PN) {
    const size_t p = idx / N, j = idx - p * N;
    const T* ph = phi + p * K * N + j;
    T s = T(0);
    for (int k = 0; k < K; ++k) s += ph[k * N] * lam[p * K + k];
    bary_log[idx] = s;
    if (b)
      for (int k = 0; k < K; ++k) b[p * K * N + k * N + j] = s - ph[k * N];
  }
}

template <typename T>
__global__ void k_exp_inplace(T* __restrict__ v, size_t n) {
  GRID_STRIDE(i, n) v[i] = d_exp<T>(v[i]);
}

// ---------------- loss (cpp/loss.h:19-90), one histogram per block ------------------
// Writes the loss gradient g into n (the dictionary recursion's start) and
// g * bary into gw (the weight recursion's start, :633-635).
template <typename T>
__global__ void k_loss(const T* __restrict__ bary, const double* __restrict__ obs,
                       const T* __restrict__ wgrad, T* __restrict__ n, T* __restrict__ gw,
                       double* __restrict__ loss, int loss_type, size_t N) {
  __shared__ double sh[32];
  const size_t p = blockIdx.x;
  double acc = 0;
  for (size_t j = threadIdx.x; j < N; j += blockDim.x) {
    const size_t i = p * N + j;
    const T v1 = bary[i];
    const double o = obs[i];
    const T v2 = (T)o;
    T g;
    if (loss_type == WDL_LOSS_TV) {
      const T d = v1 - v2;
      acc += fabs((double)v1 - o);
      g = d > T(0) ? T(0.5) : T(-0.5);
    } else if (loss_type == WDL_LOSS_QUADRATIC) {
      const double d = (double)v1 - o;
      acc += d * d;
      g = T(2) * (v1 - v2);
    } else if (loss_type == WDL_LOSS_KL) {
      const double r = (double)v1 / o;
      acc += (double)v1 * log(r > kEpsilon ? r : kEpsilon) - (double)v1 + o;
      g = safe_log<T>(v1 / v2);
    } else {  // Wasserstein: gradient precomputed by the nested Sinkhorn
      g = wgrad[i];
    }
    n[i] = g;
    gw[i] = g * v1;
  }
  acc = block_sum(acc, sh);
  if (threadIdx.x == 0 && loss_type != WDL_LOSS_WASSERSTEIN)
    loss[p] = loss_type == WDL_LOSS_TV ? 0.5 * acc : acc;
}

// Wasserstein loss helpers (cpp/loss.h:92-154): a = v1 / Kb, b = v2 / Ka.
template <typename T>
__global__ void k_ratio(const T* __restrict__ num, const double* __restrict__ num64,
                        const T* __restrict__ den, T* __restrict__ out, size_t n) {
  GRID_STRIDE(i, n) out[i] = (num ? num[i] : (T)num64[i]) / den[i];
}
template <typename T>
__global__ void k_wloss(const T* __restrict__ v1, const double* __restrict__ v2,
                        const T* __restrict__ a, const T* __restrict__ b, const T* __restrict__ c,
                        T* __restrict__ wgrad, double* __restrict__ loss, double gamma, size_t N) {
  __shared__ double sh[32];
  const size_t p = blockIdx.x;
  double acc = 0;
  for (size_t j = threadIdx.x; j < N; j += blockDim.x) {
    const size_t i = p * N + j;
    const double la = (double)safe_log<T>(a[i]), lb = (double)safe_log<T>(b[i]);
    acc += la * (double)v1[i] + lb * v2[i] - (double)a[i] * (double)c[i];
    wgrad[i] = (T)(gamma * la);
  }
  acc = block_sum(acc, sh);
  if (threadIdx.x == 0) loss[p] = gamma * acc;
}

// The reverse passes' per-(p, k) dot products are summed in two levels with a
// fixed order: blocks over kSegElems-element segments of each image write
// partial sums, k_add_partials adds them segment by segment.  The segments
// depend only on N, so a histogram's result does not depend on P or K.
constexpr size_t kSegElems = 2048;
inline size_t n_segments(size_t N) { return (N + kSegElems - 1) / kSegElems; }

__global__ void k_add_partials(double* __restrict__ dot, const double* __restrict__ part, int PK,
                               int nseg) {
  const int pk = blockIdx.x * blockDim.x + threadIdx.x;
  if (pk >= PK) return;
  double s = 0;
  for (int g = 0; g < nseg; ++g) s += part[(size_t)pk * nseg + g];
  dot[pk] += s;
}

// ---------------- kernel-domain reverse pass (:602-673), one round s ----------------
// Block per ((p, k), segment): dictionary tmp = (lambda n - v) * b[s] (when the
// dictionary recursion runs); weights dot += sum_j log(phi[s]) gw (plain log,
// as :649), u = (lambda gw - r) / phi[s].
template <typename T>
__global__ void k_bwd_pre(const T* __restrict__ n, const T* __restrict__ v,
                          const T* __restrict__ b_s, const T* __restrict__ gw,
                          const T* __restrict__ r, const T* __restrict__ phi_s,
                          const T* __restrict__ lam, T* __restrict__ tmp, T* __restrict__ u,
                          double* __restrict__ part, int K, size_t N, int dict) {
  __shared__ double sh[32];
  const size_t pk = blockIdx.x, p = pk / K;
  const T l = lam[pk];
  const size_t base = pk * N, pb = p * N;
  const size_t j0 = (size_t)blockIdx.y * kSegElems, j1 = min(N, j0 + kSegElems);
  double acc = 0;
  for (size_t j = j0 + threadIdx.x; j < j1; j += blockDim.x) {
    const size_t i = base + j;
    if (dict) tmp[i] = (l * n[pb + j] - v[i]) * b_s[i];
    const T ph = phi_s[i];
    const T g = gw[pb + j];
    acc += acc_log<T>(ph) * (double)g;
    u[i] = (l * g - r[i]) / ph;
  }
  acc = block_sum(acc, sh);
  if (threadIdx.x == 0) part[pk * gridDim.y + blockIdx.y] = acc;
}

// gradDic += c / cb[s-1]; tmp = -p c / cb^2 (dictionary recursion, when it
// runs); convu *= -p / cb^2 (:612-617, :655-660).  Thread per dictionary
// entry q = (k, j), histograms p in order: the dictionary gradient gdic[q] (KN
// doubles, summed over p here rather than kept per histogram) takes this
// round's sum over p in one update.
template <typename T>
__global__ void k_bwd_mid(const T* __restrict__ c, const T* __restrict__ cb,
                          const T* __restrict__ atoms, double* __restrict__ gdic,
                          T* __restrict__ nxt, size_t KN, int P, size_t PKN, int weights, int dict) {
  GRID_STRIDE(q, KN) {
    const T pa = atoms[q];
    double g = 0;
#pragma unroll 4
    for (int p = 0; p < P; ++p) {
      const size_t i = (size_t)p * KN + q;
      const T cbv = cb[i];
      if (dict) {
        const T cc = c[i];
        g += (double)(cc / cbv);
        nxt[i] = -pa * cc / (cbv * cbv);
      }
      if (weights) nxt[PKN + i] = c[PKN + i] * (-pa / (cbv * cbv));
    }
    if (dict) gdic[q] += g;
  }
}

// v = Kt(tmp) / phi[s-1], n = sum_k v (:619-627); r = K(convu) * b[s-1],
// gw = sum_k r (:661-669).  One thread per (p, pixel).
template <typename T>
__global__ void k_bwd_post(const T* __restrict__ c2, const T* __restrict__ phi_p,
                           const T* __restrict__ b_p, T* __restrict__ v, T* __restrict__ r,
                           T* __restrict__ n, T* __restrict__ gw, int K, size_t N, size_t PN,
                           size_t PKN, int dict) {
  GRID_STRIDE(idx, PN) {
    const size_t p = idx / N, j = idx - p * N;
    T sn = T(0), sg = T(0);
    for (int k = 0; k < K; ++k) {
      const size_t i = (p * K + k) * N + j;
      if (dict) {
        const T vv = c2[i] / phi_p[i];
        v[i] = vv;
        sn += vv;
      }
      const T rr = c2[PKN + i] * b_p[i];
      r[i] = rr;
      sg += rr;
    }
    if (dict) n[idx] = sn;
    gw[idx] = sg;
  }
}

// Round s's k_bwd_post followed by round s-1's k_bwd_pre in one pass (the
// kernel-domain counterpart of k_lbwd_post_pre below): v, r, n and gw never go
// to memory.  Block per (p, segment), one warp per atom (blockDim 32 K, K <=
// 32), two 32-pixel chunks per round, the next round's loads issued before
// this round's sums; n and gw are summed over the atoms in k order through
// SMEM (as k_bwd_post), the dot partial of (p, k) over the segment is the
// lanes' sums reduced across the warp (an order fixed by N).  dict: the
// dictionary recursion runs (v, n, tmp).
template <typename T>
struct BwdIn {
  T cv[2], cr[2], ph[2], bp[2];
};

template <typename T>
__device__ __forceinline__ void bwd_load(BwdIn<T>& in, const T* __restrict__ c2, const T* __restrict__ phi_p,
                                         const T* __restrict__ b_p, size_t ib, size_t jb, size_t j1, int jj,
                                         size_t PKN, int dict) {
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const size_t j = jb + 32 * h + jj;
    in.cv[h] = in.cr[h] = T(0);
    in.ph[h] = in.bp[h] = T(1);
    if (j < j1) {
      const size_t i = ib + j;
      if (dict) in.cv[h] = c2[i];
      in.cr[h] = c2[PKN + i];
      in.ph[h] = phi_p[i];
      in.bp[h] = b_p[i];
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(1024) k_bwd_post_pre(
    const T* __restrict__ c2, const T* __restrict__ phi_p, const T* __restrict__ b_p,
    const T* __restrict__ lam, T* __restrict__ tmp, T* __restrict__ u, double* __restrict__ part, int K,
    size_t N, size_t PKN, int dict) {
  constexpr int W = 64;  // pixels per round
  extern __shared__ __align__(16) unsigned char bwd_raw[];
  T* vs = reinterpret_cast<T*>(bwd_raw);  // [K][W]
  T* rs = vs + K * W;                     // [K][W]
  T* sums = rs + K * W;                   // [2][W]: n, gw
  const int k = threadIdx.x >> 5, jj = threadIdx.x & 31;
  const size_t p = blockIdx.x;
  const size_t j0 = (size_t)blockIdx.y * kSegElems, j1 = min(N, j0 + kSegElems);
  const T l = lam[p * K + k];
  const size_t ib = (p * K + k) * N;
  double acc = 0;
  BwdIn<T> cur, nxt;
  bwd_load(cur, c2, phi_p, b_p, ib, j0, j1, jj, PKN, dict);
  for (size_t jb = j0; jb < j1; jb += W) {
    T vv[2], rr[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      vv[h] = dict ? cur.cv[h] / cur.ph[h] : T(0);
      rr[h] = cur.cr[h] * cur.bp[h];
      if (jb + 32 * h + jj >= j1) vv[h] = rr[h] = T(0);
      vs[k * W + 32 * h + jj] = vv[h];
      rs[k * W + 32 * h + jj] = rr[h];
    }
    __syncthreads();
    if (jb + W < j1) bwd_load(nxt, c2, phi_p, b_p, ib, jb + W, j1, jj, PKN, dict);
    for (int q = threadIdx.x; q < 2 * W; q += blockDim.x) {
      if (!dict && q < W) continue;
      const T* src = q < W ? vs + q : rs + (q - W);
      T a = T(0);
      for (int kk = 0; kk < K; ++kk) a += src[kk * W];
      sums[q] = a;
    }
    __syncthreads();
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const size_t j = jb + 32 * h + jj;
      if (j < j1) {
        const size_t i = ib + j;
        const T sg = sums[W + 32 * h + jj];
        if (dict) tmp[i] = (l * sums[32 * h + jj] - vv[h]) * cur.bp[h];
        acc += acc_log<T>(cur.ph[h]) * (double)sg;
        u[i] = (l * sg - rr[h]) / cur.ph[h];
      }
    }
    __syncthreads();
    cur = nxt;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (jj == 0) part[(p * K + k) * gridDim.y + blockIdx.y] = acc;
}

// ---------------- log-domain reverse pass (:722-812), one round s -------------------
// Signed quantities are (log|x|, sign byte) pairs; sd and sw are the dictionary
// and weight recursions' sign arrays (cpp/signArray.h:24-35).
template <typename T>
__global__ void k_lbwd_pre(const T* __restrict__ n, const T* __restrict__ v,
                           const T* __restrict__ b_s, const T* __restrict__ gw,
                           const T* __restrict__ r, const T* __restrict__ phi_s,
                           const T* __restrict__ lam, T* __restrict__ tmp, T* __restrict__ u,
                           uint8_t* __restrict__ sd, uint8_t* __restrict__ sw,
                           double* __restrict__ part, int K, size_t N) {
  __shared__ double sh[32];
  const size_t pk = blockIdx.x, p = pk / K;
  const T l = lam[pk];
  const size_t base = pk * N, pb = p * N;
  const size_t j0 = (size_t)blockIdx.y * kSegElems, j1 = min(N, j0 + kSegElems);
  double acc = 0;
  for (size_t j = j0 + threadIdx.x; j < j1; j += blockDim.x) {
    const size_t i = base + j;
    const T x = l * n[pb + j] + v[i];
    sd[i] = x >= T(0);
    tmp[i] = d_log<T>(fabs(x)) + b_s[i];
    const T ph = phi_s[i];
    const T g = gw[pb + j];
    acc += (double)ph * (double)g;
    const T y = l * g + r[i];
    sw[i] = y >= T(0);
    u[i] = d_log<T>(fabs(y)) - ph;
  }
  acc = block_sum(acc, sh);
  if (threadIdx.x == 0) part[pk * gridDim.y + blockIdx.y] = acc;
}

// Thread per dictionary entry q = (k, j), histograms p in order: the
// dictionary gradient gdic[q] (KN doubles, summed over p here rather than kept
// per histogram) takes this round's sum over p in one update.
template <typename T>
__global__ void k_lbwd_mid(const T* __restrict__ c, const T* __restrict__ cb,
                           const T* __restrict__ log_atoms, const uint8_t* __restrict__ sd,
                           double* __restrict__ gdic, T* __restrict__ nxt, size_t KN, int P,
                           size_t PKN, int weights) {
  GRID_STRIDE(q, KN) {
    const T lp = log_atoms[q];
    double g = 0;
#pragma unroll 4
    for (int p = 0; p < P; ++p) {
      const size_t i = (size_t)p * KN + q;
      const T cbv = cb[i], cc = c[i];
      const T e = d_exp<T>(cc - cbv);
      g += (double)(sd[i] ? e : -e);
      nxt[i] = lp + cc - T(2) * cbv;
      if (weights) nxt[PKN + i] = c[PKN + i] + (lp - T(2) * cbv);
    }
    gdic[q] += g;
  }
}

template <typename T>
__global__ void k_lbwd_post(const T* __restrict__ c2, const T* __restrict__ phi_p,
                            const T* __restrict__ b_p, const uint8_t* __restrict__ sd,
                            const uint8_t* __restrict__ sw, T* __restrict__ v,
                            T* __restrict__ r, T* __restrict__ n, T* __restrict__ gw, int K,
                            size_t N, size_t PN, size_t PKN) {
  GRID_STRIDE(idx, PN) {
    const size_t p = idx / N, j = idx - p * N;
    T sn = T(0), sg = T(0);
    for (int k = 0; k < K; ++k) {
      const size_t i = (p * K + k) * N + j;
      T e = d_exp<T>(c2[i] - phi_p[i]);
      const T vv = sd[i] ? e : -e;
      v[i] = vv;
      sn -= vv;
      e = d_exp<T>(c2[PKN + i] + b_p[i]);
      const T rr = sw[i] ? e : -e;
      r[i] = rr;
      sg -= rr;
    }
    n[idx] = sn;
    gw[idx] = sg;
  }
}

// Round s's k_lbwd_post followed by round s-1's k_lbwd_pre in one pass: the
// post's v, r, n and gw feed only that pre, whose b and phi are the post's b_p
// and phi_p, so v, r, n and gw never go to memory.  Block per (p, segment)
// with one warp per atom (blockDim 32 K, K <= kFuseK): lane jj of warp k
// handles pixels j0 + jj + 32 m of atom k, kFuseH 32-pixel chunks per round.
// Each warp makes its atom's v and r into SMEM; the block's threads then sum n
// and gw over the atoms, one pixel and quantity per thread (k in order, as
// k_lbwd_post); each warp applies the pre to its atom.  The next round's loads
// are issued before this round's sums and pre, so they overlap them.  The dot
// partial of (p, k) over the segment is the lanes' sums reduced across the
// warp, an order fixed by N.
constexpr int kFuseK = 32, kFuseH = 2;
template <typename T>
size_t post_pre_smem(int K) { return (size_t)(2 * K + 2) * 32 * kFuseH * sizeof(T); }

template <typename T>
struct PostPreIn {  // one round's inputs of one thread
  T cv[kFuseH], cr[kFuseH], ph[kFuseH], bp[kFuseH];
  uint8_t sv[kFuseH], sr[kFuseH];
};

template <typename T>
__device__ __forceinline__ void post_pre_load(PostPreIn<T>& in, const T* __restrict__ c2,
                                              const T* __restrict__ phi_p, const T* __restrict__ b_p,
                                              const uint8_t* sd, const uint8_t* sw, size_t ib, size_t jb,
                                              size_t j1, int jj, size_t PKN) {
#pragma unroll
  for (int h = 0; h < kFuseH; ++h) {
    const size_t j = jb + 32 * h + jj;
    in.cv[h] = in.cr[h] = in.ph[h] = in.bp[h] = T(0);
    in.sv[h] = in.sr[h] = 1;
    if (j < j1) {
      const size_t i = ib + j;
      in.cv[h] = c2[i];
      in.cr[h] = c2[PKN + i];
      in.ph[h] = phi_p[i];
      in.bp[h] = b_p[i];
      in.sv[h] = sd[i];
      in.sr[h] = sw[i];
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(1024) k_lbwd_post_pre(
    const T* __restrict__ c2, const T* __restrict__ phi_p, const T* __restrict__ b_p,
    uint8_t* __restrict__ sd, uint8_t* __restrict__ sw, const T* __restrict__ lam,
    T* __restrict__ tmp, T* __restrict__ u, double* __restrict__ part, int K, size_t N, size_t PKN) {
  constexpr int W = 32 * kFuseH;  // pixels per round
  extern __shared__ __align__(16) unsigned char fuse_raw[];
  T* vs = reinterpret_cast<T*>(fuse_raw);  // [K][W] v of this round's pixels
  T* rs = vs + K * W;                      // [K][W] r
  T* sums = rs + K * W;                    // [2][W]: n, gw
  const int k = threadIdx.x >> 5, jj = threadIdx.x & 31;
  const size_t p = blockIdx.x;
  const size_t j0 = (size_t)blockIdx.y * kSegElems, j1 = min(N, j0 + kSegElems);
  const T l = lam[p * K + k];
  const size_t ib = (p * K + k) * N;
  double acc = 0;
  PostPreIn<T> cur, nxt;
  post_pre_load(cur, c2, phi_p, b_p, sd, sw, ib, j0, j1, jj, PKN);
  for (size_t jb = j0; jb < j1; jb += W) {
    T vv[kFuseH], rr[kFuseH];
#pragma unroll
    for (int h = 0; h < kFuseH; ++h) {
      T e = d_exp<T>(cur.cv[h] - cur.ph[h]);
      vv[h] = cur.sv[h] ? e : -e;
      e = d_exp<T>(cur.cr[h] + cur.bp[h]);
      rr[h] = cur.sr[h] ? e : -e;
      if (jb + 32 * h + jj >= j1) vv[h] = rr[h] = T(0);
      vs[k * W + 32 * h + jj] = vv[h];
      rs[k * W + 32 * h + jj] = rr[h];
    }
    __syncthreads();
    // the next round's inputs (the elements this thread rewrites below are this round's)
    if (jb + W < j1) post_pre_load(nxt, c2, phi_p, b_p, sd, sw, ib, jb + W, j1, jj, PKN);
    for (int q = threadIdx.x; q < 2 * W; q += blockDim.x) {
      const T* src = q < W ? vs + q : rs + (q - W);
      T a = T(0);
      for (int kk = 0; kk < K; ++kk) a -= src[kk * W];
      sums[q] = a;
    }
    __syncthreads();
#pragma unroll
    for (int h = 0; h < kFuseH; ++h) {
      const size_t j = jb + 32 * h + jj;
      if (j < j1) {
        const T sn = sums[32 * h + jj], sg = sums[W + 32 * h + jj];
        const size_t i = ib + j;
        const T x = l * sn + vv[h];
        sd[i] = x >= T(0);
        tmp[i] = d_log_mag<T>(x) + cur.bp[h];
        acc += (double)cur.ph[h] * (double)sg;
        const T y = l * sg + rr[h];
        sw[i] = y >= T(0);
        u[i] = d_log_mag<T>(y) - cur.ph[h];
      }
    }
    __syncthreads();
    cur = nxt;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (jj == 0) part[(p * K + k) * gridDim.y + blockIdx.y] = acc;
}

// ---------------- reductions and evaluate_both epilogue (:1086-1136) ----------------
// Weight part of g: (la - <w, la>) * w / scale (projection :1093-1098, chain rule
// :1125-1128, scaling :1135-1136).  One histogram per thread.
__global__ void k_project_weights(const double* __restrict__ la, const double* __restrict__ w,
                                  double* __restrict__ g, int P, int K, double scale) {
  GRID_STRIDE(p, (size_t)P) {
    double d = 0;
    for (int k = 0; k < K; ++k) d += w[p * K + k] * la[p * K + k];
    for (int k = 0; k < K; ++k) g[p * K + k] = ((la[p * K + k] - d) * w[p * K + k]) / scale;
  }
}

// Atom part of g: (G - <atom, G>) * atom (:1103-1108, :1125-1128), block per atom.
__global__ void k_project_atoms(const double* __restrict__ dic, const double* __restrict__ atoms,
                                double* __restrict__ g, size_t N) {
  __shared__ double sh[32];
  const size_t k = blockIdx.x;
  double d = 0;
  for (size_t j = threadIdx.x; j < N; j += blockDim.x) d += atoms[k * N + j] * dic[k * N + j];
  d = block_sum(d, sh);
  if (threadIdx.x == 0) sh[0] = d;
  __syncthreads();
  d = sh[0];
  for (size_t j = threadIdx.x; j < N; j += blockDim.x)
    g[k * N + j] = (dic[k * N + j] - d) * atoms[k * N + j];
}

__global__ void k_sum_losses(const double* __restrict__ loss, double* __restrict__ f, int P) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    double s = 0;
    for (int p = 0; p < P; ++p) s += loss[p];
    *f = s;
  }
}

__global__ void k_sum_over_p_f32(const float* __restrict__ gdic, double* __restrict__ out, int P,
                                 size_t KN) {
  GRID_STRIDE(i, KN) {
    double s = 0;
    for (int p = 0; p < P; ++p) s += (double)gdic[(size_t)p * KN + i];
    out[i] = s;
  }
}

// b[L] = bary[L] / phi[L] (the warm-restart store) from the fused path's tape,
// where bary = exp(acc).
__global__ void k_b_last(const float* __restrict__ acc, const float* __restrict__ phi,
                         double* __restrict__ out, int K, size_t N, size_t PKN) {
  GRID_STRIDE(i, PKN) {
    const size_t p = i / ((size_t)K * N), j = i % N;
    out[i] = (double)(expf(acc[p * N + j]) / phi[i]);
  }
}
__global__ void k_exp_to_double(const float* __restrict__ acc, double* __restrict__ out, size_t n) {
  GRID_STRIDE(i, n) out[i] = (double)expf(acc[i]);
}

// ---------------- workspace -----------------------------------------------------------
inline void alloc_into(Arena& a, void** p, size_t bytes) { *p = a.take<char>(bytes); }
inline void alloc_into(ArenaPlan& a, void** p, size_t bytes) {
  a.take<char>(bytes);
  *p = nullptr;
}

// Device workspace of one gradient_both call.  Pairs that feed one operator
// launch (buf2 = [tmp | u], cbuf2, the sign arrays sd/sw) are single
// allocations so that their halves are adjacent.
template <typename T>
struct EvalBufs {
  T *atoms, *lam, *tape_b, *tape_cb, *tape_phi, *a, *bary, *n, *gw, *buf2, *cbuf2, *v, *r, *ctmp;
  T *wa = nullptr, *wb = nullptr, *wc = nullptr, *wgrad = nullptr;
  double *atoms64, *lam64, *gdic, *dot, *loss, *dpart;
  int* range;  // [P] scalings left the FP32 range (kernel domain, FP32 forms)
  uint8_t *sd = nullptr, *sw = nullptr, *stmp = nullptr;

  template <class A>
  void layout(A& al, size_t P, size_t K, size_t L, size_t N, bool log_domain, bool wloss) {
    const size_t KN = K * N, PKN = P * KN, PN = P * N;
    auto t = [&](T*& p, size_t n) { alloc_into(al, reinterpret_cast<void**>(&p), n * sizeof(T)); };
    auto d = [&](double*& p, size_t n) { alloc_into(al, reinterpret_cast<void**>(&p), n * 8); };
    t(atoms, KN);
    t(lam, P * K);
    t(tape_b, (L + 1) * PKN);
    t(tape_cb, L * PKN);
    t(tape_phi, L * PKN);
    t(a, PKN);
    t(bary, PN);
    t(n, PN);
    t(gw, PN);
    t(buf2, 2 * PKN);
    t(cbuf2, 2 * PKN);
    t(v, PKN);
    t(r, PKN);
    t(ctmp, 2 * PKN);
    d(atoms64, KN);
    d(lam64, P * K);
    d(gdic, PKN);
    d(dot, P * K);
    d(dpart, P * K * n_segments(N));
    d(loss, P);
    alloc_into(al, reinterpret_cast<void**>(&range), P * sizeof(int));
    if (wloss) {
      t(wa, PN);
      t(wb, PN);
      t(wc, PN);
      t(wgrad, PN);
    }
    if (log_domain) {
      alloc_into(al, reinterpret_cast<void**>(&sd), 2 * PKN);
      alloc_into(al, reinterpret_cast<void**>(&stmp), 2 * PKN);
      sw = sd ? sd + PKN : nullptr;
    }
  }
};

template <typename T>
size_t eval_bytes_t(size_t P, size_t K, size_t L, size_t N, bool log_domain, bool wloss) {
  ArenaPlan plan;
  EvalBufs<T> b;
  b.layout(plan, P, K, L, N, log_domain, wloss);
  return plan.off + 256;
}

int launch_cfg(wdl_ctx* ctx, size_t n) { return grid_for(n, 256, ctx->sm_count, 8); }

// Nested Sinkhorn of the Wasserstein loss (cpp/loss.h:92-154) on all P
// barycenters at once, kernel domain, 50 inner iterations.
template <typename T>
int wasserstein_loss(wdl_ctx* ctx, EvalBufs<T>& B, const double* obs, int P, cudaStream_t s) {
  const size_t N = ctx->N, PN = (size_t)P * N;
  const unsigned G = launch_cfg(ctx, PN);
  int rc;
  k_fill<T><<<G, 256, 0, s>>>(B.wb, T(1), PN);
  WDL_LAUNCH_CHECK(ctx);
  for (int it = 0; it < 50; ++it) {
    if ((rc = conv_stack<T>(ctx, B.wb, B.wc, B.ctmp, P, s))) return rc;
    k_ratio<T><<<G, 256, 0, s>>>(B.bary, nullptr, B.wc, B.wa, PN);
    WDL_LAUNCH_CHECK(ctx);
    if ((rc = conv_stack<T>(ctx, B.wa, B.wc, B.ctmp, P, s))) return rc;
    k_ratio<T><<<G, 256, 0, s>>>(nullptr, obs, B.wc, B.wb, PN);
    WDL_LAUNCH_CHECK(ctx);
  }
  if ((rc = conv_stack<T>(ctx, B.wb, B.wc, B.ctmp, P, s))) return rc;
  k_wloss<T><<<P, 256, 0, s>>>(B.bary, obs, B.wa, B.wb, B.wc, B.wgrad, B.loss, ctx->gamma, N);
  WDL_LAUNCH_CHECK(ctx);
  return WDL_OK;
}

template <typename T>
int gradient_both_t(wdl_ctx* ctx, int P, int K, int L, int loss_type, const double* atoms,
                    const double* weights, const double* observed, const double* b_init,
                    double* result_la, double* result_dic, double* bary_out, double* loss_out,
                    double* b_last, cudaStream_t s, bool normalise) {
  const bool log_domain = ctx->domain == WDL_DOMAIN_LOG;
  const bool wloss = loss_type == WDL_LOSS_WASSERSTEIN;
  const size_t N = ctx->N, KN = (size_t)K * N, PKN = (size_t)P * KN, PN = (size_t)P * N;
  int rc;
  if ((rc = ensure_arena(ctx, eval_bytes_t<T>(P, K, L, N, log_domain, wloss)))) return rc;
  ctx->arena.reset();
  EvalBufs<T> B;
  B.layout(ctx->arena, P, K, L, N, log_domain, wloss);
  const unsigned G_PKN = launch_cfg(ctx, PKN), G_PN = launch_cfg(ctx, PN),
                 G_2PKN = launch_cfg(ctx, 2 * PKN);

  // Inputs: normalised FP64 copies (normalize_values, :562) and their T casts.
  if (normalise) {
    k_normalise_rows<<<K, 256, 0, s>>>(atoms, B.atoms64, N, 0.0);
    WDL_LAUNCH_CHECK(ctx);
    k_normalise_rows<<<P, 32, 0, s>>>(weights, B.lam64, K, 0.0);
    WDL_LAUNCH_CHECK(ctx);
  } else {
    WDL_CUDA_TRY(ctx, cudaMemcpyAsync(B.atoms64, atoms, KN * 8, cudaMemcpyDeviceToDevice, s));
    WDL_CUDA_TRY(ctx, cudaMemcpyAsync(B.lam64, weights, (size_t)P * K * 8, cudaMemcpyDeviceToDevice, s));
  }
  if (log_domain) k_log_of<T><<<launch_cfg(ctx, KN), 256, 0, s>>>(B.atoms64, B.atoms, KN);
  else k_cast<T><<<launch_cfg(ctx, KN), 256, 0, s>>>(B.atoms64, B.atoms, KN);
  WDL_LAUNCH_CHECK(ctx);
  k_cast<T><<<1, 256, 0, s>>>(B.lam64, B.lam, (size_t)P * K);
  WDL_LAUNCH_CHECK(ctx);
  if (b_init) {
    if (log_domain) k_log_of<T><<<G_PKN, 256, 0, s>>>(b_init, B.tape_b, PKN);
    else k_cast<T><<<G_PKN, 256, 0, s>>>(b_init, B.tape_b, PKN);
  } else {
    k_fill<T><<<G_PKN, 256, 0, s>>>(B.tape_b, log_domain ? T(0) : T(1), PKN);
  }
  WDL_LAUNCH_CHECK(ctx);

  // Forward Bregman projections, storing b, conv_b and phi (:565-593 / :700-720).
  int* range = (!log_domain && sizeof(T) == 4) ? B.range : nullptr;
  if (range) WDL_CUDA_TRY(ctx, cudaMemsetAsync(range, 0, (size_t)P * sizeof(int), s));
  for (int it = 1; it <= L; ++it) {
    const T* b_prev = B.tape_b + (size_t)(it - 1) * PKN;
    T* cb = B.tape_cb + (size_t)(it - 1) * PKN;
    T* phi = B.tape_phi + (size_t)(it - 1) * PKN;
    T* b_next = B.tape_b + (size_t)it * PKN;
    if (!log_domain) {
      if ((rc = conv_stack<T>(ctx, b_prev, cb, B.ctmp, (size_t)P * K, s))) return rc;
      k_div_atoms<T><<<G_PKN, 256, 0, s>>>(B.atoms, cb, B.a, KN, PKN, range);
      WDL_LAUNCH_CHECK(ctx);
      if ((rc = conv_stack<T>(ctx, B.a, phi, B.ctmp, (size_t)P * K, s))) return rc;
      k_bary_b<T><<<G_PN, 256, 0, s>>>(phi, B.lam64, b_next, B.bary, K, N, PN, range);
    } else {
      // cb = conv(b_prev), and a = log atoms - cb from the same pass
      if ((rc = log_conv_stack<T>(ctx, b_prev, cb, B.ctmp, (size_t)P * K, nullptr, nullptr,
                                  nullptr, s, B.atoms, B.a, KN)))
        return rc;
      if ((rc = log_conv_stack<T>(ctx, B.a, phi, B.ctmp, (size_t)P * K, nullptr, nullptr,
                                  nullptr, s)))
        return rc;
      k_log_bary_b<T><<<G_PN, 256, 0, s>>>(phi, B.lam, b_next, B.bary, K, N, PN);
    }
    WDL_LAUNCH_CHECK(ctx);
  }
  if (log_domain) {
    k_exp_inplace<T><<<G_PN, 256, 0, s>>>(B.bary, PN);
    WDL_LAUNCH_CHECK(ctx);
  }
  if (range) {
    k_poison_out_of_range<T><<<G_PN, 256, 0, s>>>(B.bary, range, N, PN);
    WDL_LAUNCH_CHECK(ctx);
  }

  // Loss and its gradient (:597).
  if (wloss && (rc = wasserstein_loss<T>(ctx, B, observed, P, s))) return rc;
  k_loss<T><<<P, 256, 0, s>>>(B.bary, observed, B.wgrad, B.n, B.gw, B.loss, loss_type, N);
  WDL_LAUNCH_CHECK(ctx);

  // Reverse pass, both recursions per round (:602-673 / :730-812).  With no
  // dictionary gradient requested, the kernel domain runs the weight
  // recursion alone: the operator takes only the second half of each
  // [dictionary | weights] image pair.
  const int dict = (result_dic || log_domain) ? 1 : 0;
  WDL_CUDA_TRY(ctx, cudaMemsetAsync(B.v, 0, PKN * sizeof(T), s));
  WDL_CUDA_TRY(ctx, cudaMemsetAsync(B.r, 0, PKN * sizeof(T), s));
  // the dictionary gradient is summed over p as it goes (KN entries)
  WDL_CUDA_TRY(ctx, cudaMemsetAsync(B.gdic, 0, KN * sizeof(double), s));
  WDL_CUDA_TRY(ctx, cudaMemsetAsync(B.dot, 0, (size_t)P * K * sizeof(double), s));
  T* tmp = B.buf2;
  T* u = B.buf2 + PKN;
  for (int sstep = L; sstep >= 1; --sstep) {
    const T* b_s = B.tape_b + (size_t)sstep * PKN;
    const T* phi_s = B.tape_phi + (size_t)(sstep - 1) * PKN;
    const T* cb_p = B.tape_cb + (size_t)(sstep - 1) * PKN;
    const bool more = sstep > 1;
    const size_t nimg = (size_t)(more ? 2 : 1) * P * K;
    if (!log_domain) {
      // the first round's pre here; later rounds' pre ran with the previous post
      if (sstep == L || K > kFuseK) {
        k_bwd_pre<T><<<dim3((unsigned)(P * K), (unsigned)n_segments(N)), 256, 0, s>>>(
            B.n, B.v, b_s, B.gw, B.r, phi_s, B.lam, tmp, u, B.dpart, K, N, dict);
        WDL_LAUNCH_CHECK(ctx);
      }
      k_add_partials<<<(P * K + 127) / 128, 128, 0, s>>>(B.dot, B.dpart, P * K, (int)n_segments(N));
      WDL_LAUNCH_CHECK(ctx);
      if (dict) {
        if ((rc = conv_stack<T>(ctx, B.buf2, B.cbuf2, B.ctmp, nimg, s))) return rc;
      } else if (more) {
        if ((rc = conv_stack<T>(ctx, u, B.cbuf2 + PKN, B.ctmp, (size_t)P * K, s))) return rc;
      }
      if (dict || more) {
        k_bwd_mid<T><<<launch_cfg(ctx, KN), 256, 0, s>>>(B.cbuf2, cb_p, B.atoms, B.gdic, B.buf2, KN, P, PKN,
                                                       more, dict);
        WDL_LAUNCH_CHECK(ctx);
      }
      if (!more) break;
      if (dict) {
        if ((rc = conv_stack<T>(ctx, B.buf2, B.cbuf2, B.ctmp, nimg, s))) return rc;
      } else {
        if ((rc = conv_stack<T>(ctx, u, B.cbuf2 + PKN, B.ctmp, (size_t)P * K, s))) return rc;
      }
      const T* phi_p = B.tape_phi + (size_t)(sstep - 2) * PKN;
      const T* b_p = B.tape_b + (size_t)(sstep - 1) * PKN;
      if (K <= kFuseK) {
        k_bwd_post_pre<T><<<dim3((unsigned)P, (unsigned)n_segments(N)), 32 * K,
                            (size_t)(2 * K + 2) * 64 * sizeof(T), s>>>(B.cbuf2, phi_p, b_p, B.lam, tmp, u,
                                                                       B.dpart, K, N, PKN, dict);
      } else {
        k_bwd_post<T><<<G_PN, 256, 0, s>>>(B.cbuf2, phi_p, b_p, B.v, B.r, B.n, B.gw, K, N, PN, PKN, dict);
      }
      WDL_LAUNCH_CHECK(ctx);
    } else {
      // the first round's pre here; later rounds' pre ran with the previous post
      if (sstep == L || K > kFuseK) {
        k_lbwd_pre<T><<<dim3((unsigned)(P * K), (unsigned)n_segments(N)), 256, 0, s>>>(
            B.n, B.v, b_s, B.gw, B.r, phi_s, B.lam, tmp, u, B.sd, B.sw, B.dpart, K, N);
        WDL_LAUNCH_CHECK(ctx);
      }
      k_add_partials<<<(P * K + 127) / 128, 128, 0, s>>>(B.dot, B.dpart, P * K, (int)n_segments(N));
      WDL_LAUNCH_CHECK(ctx);
      // sd and sw are adjacent, so the pair is one 2*P*K-image signed operand.
      if ((rc = log_conv_stack<T>(ctx, B.buf2, B.cbuf2, B.ctmp, nimg, B.sd, B.sd, B.stmp, s)))
        return rc;
      k_lbwd_mid<T><<<launch_cfg(ctx, KN), 256, 0, s>>>(B.cbuf2, cb_p, B.atoms, B.sd, B.gdic, B.buf2,
                                                        KN, P, PKN, more);
      WDL_LAUNCH_CHECK(ctx);
      if (!more) break;
      if ((rc = log_conv_stack<T>(ctx, B.buf2, B.cbuf2, B.ctmp, nimg, B.sd, B.sd, B.stmp, s)))
        return rc;
      const T* phi_p = B.tape_phi + (size_t)(sstep - 2) * PKN;
      const T* b_p = B.tape_b + (size_t)(sstep - 1) * PKN;
      if (K <= kFuseK) {
        const size_t smem = post_pre_smem<T>(K);
        if (smem > 48 * 1024)
          cudaFuncSetAttribute(k_lbwd_post_pre<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k_lbwd_post_pre<T><<<dim3((unsigned)P, (unsigned)n_segments(N)), 32 * K, smem, s>>>(
            B.cbuf2, phi_p, b_p, B.sd, B.sw, B.lam, tmp, u, B.dpart, K, N, PKN);
      } else {
        k_lbwd_post<T><<<G_PN, 256, 0, s>>>(B.cbuf2, phi_p, b_p, B.sd, B.sw, B.v, B.r, B.n, B.gw,
                                            K, N, PN, PKN);
      }
      WDL_LAUNCH_CHECK(ctx);
    }
  }

  // Outputs.
  WDL_CUDA_TRY(ctx, cudaMemcpyAsync(result_la, B.dot, (size_t)P * K * 8, cudaMemcpyDeviceToDevice, s));
  if (result_dic)
    WDL_CUDA_TRY(ctx, cudaMemcpyAsync(result_dic, B.gdic, KN * sizeof(double), cudaMemcpyDeviceToDevice, s));
  if (bary_out) {
    k_cast_back<T><<<G_PN, 256, 0, s>>>(B.bary, bary_out, PN);
    WDL_LAUNCH_CHECK(ctx);
  }
  if (loss_out) WDL_CUDA_TRY(ctx, cudaMemcpyAsync(loss_out, B.loss, (size_t)P * 8, cudaMemcpyDeviceToDevice, s));
  if (b_last) {
    const T* bl = B.tape_b + (size_t)L * PKN;
    if (log_domain) {
      return set_error(ctx, WDL_ERR_UNSUPPORTED, "warm restart store is kernel-domain only (as the reference)");
    }
    k_cast_back<T><<<G_PKN, 256, 0, s>>>(bl, b_last, PKN);
    WDL_LAUNCH_CHECK(ctx);
  }
  return WDL_OK;
}

// Forward-only barycenter for P weight vectors (cpp/inverseWasserstein.h:115-201).
template <typename T>
int barycenter_t(wdl_ctx* ctx, int P, int K, int L, const double* atoms, const double* weights,
                 double* bary_out, cudaStream_t s) {
  const bool log_domain = ctx->domain == WDL_DOMAIN_LOG;
  const size_t N = ctx->N, KN = (size_t)K * N, PKN = (size_t)P * KN, PN = (size_t)P * N;
  int rc;
  if ((rc = ensure_arena(ctx, barycenter_bytes(ctx, P, K)))) return rc;
  ctx->arena.reset();
  Arena& A = ctx->arena;
  double* atoms64 = A.take<double>(KN);
  double* lam64 = A.take<double>((size_t)P * K);
  T* at = A.take<T>(KN);
  T* lam = A.take<T>((size_t)P * K);
  T* b = A.take<T>(PKN);
  T* conv = A.take<T>(PKN);
  T* a = A.take<T>(PKN);
  T* tmp = A.take<T>(PKN);
  T* bary = A.take<T>(PN);
  int* range = (!log_domain && sizeof(T) == 4) ? A.take<int>((size_t)P) : nullptr;
  if (range) WDL_CUDA_TRY(ctx, cudaMemsetAsync(range, 0, (size_t)P * sizeof(int), s));
  k_normalise_rows<<<K, 256, 0, s>>>(atoms, atoms64, N, 0.0);
  WDL_LAUNCH_CHECK(ctx);
  k_normalise_rows<<<P, 32, 0, s>>>(weights, lam64, K, 0.0);
  WDL_LAUNCH_CHECK(ctx);
  if (log_domain) k_log_of<T><<<launch_cfg(ctx, KN), 256, 0, s>>>(atoms64, at, KN);
  else k_cast<T><<<launch_cfg(ctx, KN), 256, 0, s>>>(atoms64, at, KN);
  WDL_LAUNCH_CHECK(ctx);
  k_cast<T><<<1, 256, 0, s>>>(lam64, lam, (size_t)P * K);
  WDL_LAUNCH_CHECK(ctx);
  k_fill<T><<<launch_cfg(ctx, PKN), 256, 0, s>>>(b, log_domain ? T(0) : T(1), PKN);
  WDL_LAUNCH_CHECK(ctx);
  for (int it = 0; it < L; ++it) {
    if (!log_domain) {
      if ((rc = conv_stack<T>(ctx, b, conv, tmp, (size_t)P * K, s))) return rc;
      k_div_atoms<T><<<launch_cfg(ctx, PKN), 256, 0, s>>>(at, conv, a, KN, PKN, range);
      WDL_LAUNCH_CHECK(ctx);
      if ((rc = conv_stack<T>(ctx, a, conv, tmp, (size_t)P * K, s))) return rc;
      k_bary_b<T><<<launch_cfg(ctx, PN), 256, 0, s>>>(conv, lam64, b, bary, K, N, PN, range);
    } else {
      if ((rc = log_conv_stack<T>(ctx, b, conv, tmp, (size_t)P * K, nullptr, nullptr, nullptr, s, at, a,
                                  KN)))
        return rc;
      if ((rc = log_conv_stack<T>(ctx, a, conv, tmp, (size_t)P * K, nullptr, nullptr, nullptr, s)))
        return rc;
      k_log_bary_b<T><<<launch_cfg(ctx, PN), 256, 0, s>>>(conv, lam, b, bary, K, N, PN);
    }
    WDL_LAUNCH_CHECK(ctx);
  }
  if (log_domain) {
    k_exp_inplace<T><<<launch_cfg(ctx, PN), 256, 0, s>>>(bary, PN);
    WDL_LAUNCH_CHECK(ctx);
  }
  if (range) {
    k_poison_out_of_range<T><<<launch_cfg(ctx, PN), 256, 0, s>>>(bary, range, N, PN);
    WDL_LAUNCH_CHECK(ctx);
  }
  k_cast_back<T><<<launch_cfg(ctx, PN), 256, 0, s>>>(bary, bary_out, PN);
  WDL_LAUNCH_CHECK(ctx);
  return WDL_OK;
}

// Fused tensor-core path: one persistent kernel for forward, loss and reverse
// pass (sinkhorn_tc.cu).  Inputs are normalised here in FP64 as above.
struct FusedBufs {
  double *atoms64, *lam64, *dot, *loss;
  float *atoms, *lam, *b0, *cb, *phi, *acc, *nb, *gwb, *v, *r, *gdic;
  int* sync;       // work, err, then done_fwd/bary_ready/done_bwd/msg_ready/range [5P]
  SkProblem* prob; // device copy of the problem descriptor
  template <class A>
  void layout(A& al, size_t P, size_t K, size_t L, size_t N, bool b_init, bool fwd_only) {
    const size_t KN = K * N, PKN = P * KN, PN = P * N, slots = fwd_only ? 2 : L;
    auto f = [&](float*& p, size_t n) { alloc_into(al, reinterpret_cast<void**>(&p), n * 4); };
    auto d = [&](double*& p, size_t n) { alloc_into(al, reinterpret_cast<void**>(&p), n * 8); };
    d(atoms64, KN);
    d(lam64, P * K);
    d(dot, P * K);
    d(loss, P);
    f(atoms, KN);
    f(lam, P * K);
    b0 = nullptr;
    if (b_init) f(b0, PKN);
    f(cb, fwd_only ? 1 : slots * PKN);
    f(phi, slots * PKN);
    f(acc, slots * PN);
    f(nb, fwd_only ? 1 : 2 * PN);
    f(gwb, fwd_only ? 1 : 2 * PN);
    f(v, fwd_only ? 1 : PKN);
    f(r, fwd_only ? 1 : PKN);
    f(gdic, fwd_only ? 1 : PKN);
    alloc_into(al, reinterpret_cast<void**>(&sync), (2 + 5 * P) * sizeof(int));
    alloc_into(al, reinterpret_cast<void**>(&prob), sizeof(SkProblem));
  }
};

size_t fused_bytes(size_t P, size_t K, size_t L, size_t N, bool b_init, bool fwd_only) {
  ArenaPlan plan;
  FusedBufs b;
  b.layout(plan, P, K, L, N, b_init, fwd_only);
  return plan.off + 256;
}

bool use_fused(const wdl_ctx* ctx, int loss_type) {
  return tc_fused(ctx) && ctx->domain == WDL_DOMAIN_KERNEL && loss_type != WDL_LOSS_WASSERSTEIN;
}

int prepare_fused(wdl_ctx* ctx, FusedBufs& B, int P, int K, const double* atoms,
                  const double* weights, const double* b_init, bool normalise, cudaStream_t s) {
  const size_t N = ctx->N, KN = (size_t)K * N, PKN = (size_t)P * KN;
  if (normalise) {
    k_normalise_rows<<<K, 256, 0, s>>>(atoms, B.atoms64, N, 0.0);
    WDL_LAUNCH_CHECK(ctx);
    k_normalise_rows<<<P, 32, 0, s>>>(weights, B.lam64, K, 0.0);
    WDL_LAUNCH_CHECK(ctx);
  } else {
    WDL_CUDA_TRY(ctx, cudaMemcpyAsync(B.atoms64, atoms, KN * 8, cudaMemcpyDeviceToDevice, s));
    WDL_CUDA_TRY(ctx, cudaMemcpyAsync(B.lam64, weights, (size_t)P * K * 8, cudaMemcpyDeviceToDevice, s));
  }
  k_cast<float><<<launch_cfg(ctx, KN), 256, 0, s>>>(B.atoms64, B.atoms, KN);
  WDL_LAUNCH_CHECK(ctx);
  k_cast<float><<<1, 256, 0, s>>>(B.lam64, B.lam, (size_t)P * K);
  WDL_LAUNCH_CHECK(ctx);
  if (b_init) {
    k_cast<float><<<launch_cfg(ctx, PKN), 256, 0, s>>>(b_init, B.b0, PKN);
    WDL_LAUNCH_CHECK(ctx);
  }
  return WDL_OK;
}

// Fills the problem descriptor, copies it to the device and launches.
int launch_single(wdl_ctx* ctx, const FusedBufs& B, int P, int K, int L, int loss_type,
                  const double* obs, bool fwd_only, bool need_dic, cudaStream_t s) {
  SkProblem pr{};
  sk_fill_geometry(pr, ctx->W, ctx->H, ctx->precision == WDL_SPLIT_BF16);
  pr.K = K;
  pr.L = L;
  pr.P = P;
  pr.loss_type = loss_type;
  pr.fwd_only = fwd_only ? 1 : 0;
  pr.need_dic = need_dic ? 1 : 0;
  pr.atoms = B.atoms;
  pr.lam = B.lam;
  pr.obs = obs;
  pr.b0 = B.b0;
  pr.cb = B.cb;
  pr.phi = B.phi;
  pr.acc = B.acc;
  pr.nb = B.nb;
  pr.gwb = B.gwb;
  pr.v = B.v;
  pr.r = B.r;
  pr.gdic = B.gdic;
  pr.dot = B.dot;
  pr.loss = B.loss;
  pr.sync = B.sync + 2;
  // Pageable source: the copy is staged before the call returns.
  WDL_CUDA_TRY(ctx, cudaMemcpyAsync(B.prob, &pr, sizeof(pr), cudaMemcpyHostToDevice, s));
  SkArgs a{};
  a.G = ctx->G32[ctx->W >= ctx->H ? 0 : 1];
  a.Gn = ctx->W >= ctx->H ? ctx->W : ctx->H;
  a.nprobs = 1;
  a.probs = B.prob;
  a.items = nullptr;
  a.total = (long long)sk_problem_items(pr);
  a.apps = sk_problem_applications(pr);
  a.sync = B.sync;
  int rc;
  if ((rc = sinkhorn_tc_launch(ctx, a, s))) return rc;
  ctx->fused_sync = B.sync;
  return WDL_OK;
}

int gradient_both_fused(wdl_ctx* ctx, int P, int K, int L, int loss_type, const double* atoms,
                        const double* weights, const double* observed, const double* b_init,
                        double* result_la, double* result_dic, double* bary_out, double* loss_out,
                        double* b_last, cudaStream_t s, bool normalise) {
  const size_t N = ctx->N, KN = (size_t)K * N, PKN = (size_t)P * KN, PN = (size_t)P * N;
  int rc;
  if ((rc = ensure_arena(ctx, fused_bytes(P, K, L, N, b_init != nullptr, false)))) return rc;
  ctx->arena.reset();
  FusedBufs B;
  B.layout(ctx->arena, P, K, L, N, b_init != nullptr, false);
  if ((rc = prepare_fused(ctx, B, P, K, atoms, weights, b_init, normalise, s))) return rc;
  WDL_CUDA_TRY(ctx, cudaMemsetAsync(B.v, 0, PKN * 4, s));
  WDL_CUDA_TRY(ctx, cudaMemsetAsync(B.r, 0, PKN * 4, s));
  WDL_CUDA_TRY(ctx, cudaMemsetAsync(B.gdic, 0, PKN * 4, s));
  WDL_CUDA_TRY(ctx, cudaMemsetAsync(B.dot, 0, (size_t)P * K * 8, s));
  WDL_CUDA_TRY(ctx, cudaMemsetAsync(B.acc, 0, (size_t)L * PN * 4, s));
  WDL_CUDA_TRY(ctx, cudaMemsetAsync(B.nb, 0, 2 * PN * 4, s));
  WDL_CUDA_TRY(ctx, cudaMemsetAsync(B.gwb, 0, 2 * PN * 4, s));
  if ((rc = launch_single(ctx, B, P, K, L, loss_type, observed, false, result_dic != nullptr, s)))
    return rc;
  WDL_CUDA_TRY(ctx, cudaMemcpyAsync(result_la, B.dot, (size_t)P * K * 8, cudaMemcpyDeviceToDevice, s));
  if (result_dic) {
    k_sum_over_p_f32<<<launch_cfg(ctx, KN), 256, 0, s>>>(B.gdic, result_dic, P, KN);
    WDL_LAUNCH_CHECK(ctx);
  }
  const float* acc_L = B.acc + (size_t)(L - 1) * PN;
  if (bary_out) {
    k_exp_to_double<<<launch_cfg(ctx, PN), 256, 0, s>>>(acc_L, bary_out, PN);
    WDL_LAUNCH_CHECK(ctx);
  }
  if (loss_out) WDL_CUDA_TRY(ctx, cudaMemcpyAsync(loss_out, B.loss, (size_t)P * 8, cudaMemcpyDeviceToDevice, s));
  if (b_last) {
    k_b_last<<<launch_cfg(ctx, PKN), 256, 0, s>>>(acc_L, B.phi + (size_t)(L - 1) * PKN, b_last, K, N, PKN);
    WDL_LAUNCH_CHECK(ctx);
  }
  return WDL_OK;
}

int barycenter_fused(wdl_ctx* ctx, int P, int K, int L, const double* atoms, const double* weights,
                     double* bary_out, cudaStream_t s) {
  const size_t N = ctx->N, PN = (size_t)P * N;
  int rc;
  if ((rc = ensure_arena(ctx, fused_bytes(P, K, L, N, false, true)))) return rc;
  ctx->arena.reset();
  FusedBufs B;
  B.layout(ctx->arena, P, K, L, N, false, true);
  if ((rc = prepare_fused(ctx, B, P, K, atoms, weights, nullptr, true, s))) return rc;
  WDL_CUDA_TRY(ctx, cudaMemsetAsync(B.acc, 0, 2 * PN * 4, s));
  if ((rc = launch_single(ctx, B, P, K, L, WDL_LOSS_QUADRATIC, nullptr, true, false, s))) return rc;
  k_exp_to_double<<<launch_cfg(ctx, PN), 256, 0, s>>>(B.acc + (size_t)((L - 1) & 1) * PN, bary_out, PN);
  WDL_LAUNCH_CHECK(ctx);
  return WDL_OK;
}

bool use_fp64(const wdl_ctx* ctx) { return ctx->precision == WDL_FP64; }

}  // namespace

size_t eval_bytes(const wdl_ctx* ctx, int P, int K, int L) {
  const bool log_domain = ctx->domain == WDL_DOMAIN_LOG;
  if (tc_fused(ctx) && !log_domain) {
    const size_t a = fused_bytes(P, K, L, ctx->N, true, false);
    const size_t b = eval_bytes_t<float>(P, K, L, ctx->N, false, true);  // Wasserstein loss runs unfused
    return a > b ? a : b;
  }
  return use_fp64(ctx) ? eval_bytes_t<double>(P, K, L, ctx->N, log_domain, true)
                       : eval_bytes_t<float>(P, K, L, ctx->N, log_domain, true);
}

size_t barycenter_bytes(const wdl_ctx* ctx, int P, int K) {
  if (tc_fused(ctx) && ctx->domain == WDL_DOMAIN_KERNEL) return fused_bytes(P, K, 2, ctx->N, false, true);
  const size_t N = ctx->N, KN = (size_t)K * N, PKN = (size_t)P * KN, PN = (size_t)P * N;
  const size_t t = use_fp64(ctx) ? 8 : 4;
  return 8 * (KN + (size_t)P * K) + t * (KN + (size_t)P * K + 4 * PKN + PN) + 4 * (size_t)P + 17 * 256;
}

// The CUDA-core path issues ~7 launches per iteration and reverse step (about
// 800 for L = 60); an L-BFGS loop repeats the same call with the same buffers.
// The first call with a given key runs eagerly (the workspace settles), the
// second is captured into a CUDA graph, later ones replay it.  The key holds
// every size, pointer and the stream, plus the workspace base and size, so a
// replay touches exactly the memory an eager call would.
int replay_or_run(wdl_ctx* ctx, const unsigned long long (&key)[20], cudaStream_t s,
                  const std::function<int()>& run) {
  if (ctx->profiling || ctx->trace_level || s == nullptr || s == cudaStreamLegacy ||
      s == cudaStreamPerThread)
    return run();
  // inside a caller's own capture the call becomes part of that graph
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cap) != cudaSuccess || cap != cudaStreamCaptureStatusNone) return run();
  wdl_ctx::GraphEntry* e = nullptr;
  for (auto& g : ctx->graphs)
    if (!std::memcmp(g.key, key, sizeof(key))) e = &g;
  if (e && e->exec) {
    ctx->launches += e->launches;
    WDL_CUDA_TRY(ctx, cudaGraphLaunch(e->exec, s));
    return WDL_OK;
  }
  if (!e) {  // first sighting: eager
    const int rc = run();
    if (rc) return rc;
    if (ctx->graphs.size() >= 16) {
      if (ctx->graphs.front().exec) cudaGraphExecDestroy(ctx->graphs.front().exec);
      ctx->graphs.erase(ctx->graphs.begin());
    }
    ctx->graphs.emplace_back();
    std::memcpy(ctx->graphs.back().key, key, sizeof(key));
    ctx->graphs.back().seen = 1;
    return WDL_OK;
  }
  // second sighting: capture, instantiate, launch
  const long long l0 = ctx->launches;
  WDL_CUDA_TRY(ctx, cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed));
  const int rc = run();
  cudaGraph_t graph = nullptr;
  const cudaError_t ce = cudaStreamEndCapture(s, &graph);
  if (rc) {
    if (graph) cudaGraphDestroy(graph);
    return rc;
  }
  if (ce != cudaSuccess) return cuda_error(ctx, ce, "cudaStreamEndCapture");
  const cudaError_t ie = cudaGraphInstantiate(&e->exec, graph, 0);
  cudaGraphDestroy(graph);
  if (ie != cudaSuccess) {
    e->exec = nullptr;
    return cuda_error(ctx, ie, "cudaGraphInstantiate");
  }
  e->launches = ctx->launches - l0;
  WDL_CUDA_TRY(ctx, cudaGraphLaunch(e->exec, s));
  return WDL_OK;
}

int gradient_both_dev(wdl_ctx* ctx, int P, int K, int L, int loss_type, const double* atoms,
                      const double* weights, const double* observed, const double* b_init,
                      double* result_la, double* result_dic, double* bary, double* loss,
                      double* b_last, cudaStream_t s, bool normalise) {
  if (use_fused(ctx, loss_type))
    return gradient_both_fused(ctx, P, K, L, loss_type, atoms, weights, observed, b_init, result_la,
                               result_dic, bary, loss, b_last, s, normalise);
  // the workspace is sized before the key is formed, so a replay never needs
  // a larger one
  const bool f64 = use_fp64(ctx);
  const bool log_domain = ctx->domain == WDL_DOMAIN_LOG;
  const size_t need = f64 ? eval_bytes_t<double>(P, K, L, ctx->N, log_domain, loss_type == WDL_LOSS_WASSERSTEIN)
                          : eval_bytes_t<float>(P, K, L, ctx->N, log_domain, loss_type == WDL_LOSS_WASSERSTEIN);
  int rc;
  if ((rc = ensure_arena(ctx, need))) return rc;
  const unsigned long long key[20] = {
      1ull, (unsigned long long)P, (unsigned long long)K, (unsigned long long)L,
      (unsigned long long)loss_type, (unsigned long long)normalise,
      (unsigned long long)(uintptr_t)atoms, (unsigned long long)(uintptr_t)weights,
      (unsigned long long)(uintptr_t)observed, (unsigned long long)(uintptr_t)b_init,
      (unsigned long long)(uintptr_t)result_la, (unsigned long long)(uintptr_t)result_dic,
      (unsigned long long)(uintptr_t)bary, (unsigned long long)(uintptr_t)loss,
      (unsigned long long)(uintptr_t)b_last, (unsigned long long)(uintptr_t)s,
      (unsigned long long)(uintptr_t)ctx->arena.ptr, (unsigned long long)ctx->arena.bytes, 0ull, 0ull};
  return replay_or_run(ctx, key, s, [&]() {
    if (f64)
      return gradient_both_t<double>(ctx, P, K, L, loss_type, atoms, weights, observed, b_init,
                                     result_la, result_dic, bary, loss, b_last, s, normalise);
    return gradient_both_t<float>(ctx, P, K, L, loss_type, atoms, weights, observed, b_init,
                                  result_la, result_dic, bary, loss, b_last, s, normalise);
  });
}

int barycenter_dev(wdl_ctx* ctx, int P, int K, int L, const double* atoms, const double* weights,
                   double* bary, cudaStream_t s) {
  if (use_fused(ctx, WDL_LOSS_QUADRATIC)) return barycenter_fused(ctx, P, K, L, atoms, weights, bary, s);
  // replayed like gradient_both_dev (a request loop repeats the same call);
  // the workspace is sized before the key is formed
  int rc;
  if ((rc = ensure_arena(ctx, barycenter_bytes(ctx, P, K)))) return rc;
  const unsigned long long key[20] = {
      2ull, (unsigned long long)P, (unsigned long long)K, (unsigned long long)L, 0ull, 0ull,
      (unsigned long long)(uintptr_t)atoms, (unsigned long long)(uintptr_t)weights, 0ull, 0ull,
      (unsigned long long)(uintptr_t)bary, 0ull, 0ull, 0ull, 0ull, (unsigned long long)(uintptr_t)s,
      (unsigned long long)(uintptr_t)ctx->arena.ptr, (unsigned long long)ctx->arena.bytes, 0ull, 0ull};
  return replay_or_run(ctx, key, s, [&]() {
    if (use_fp64(ctx)) return barycenter_t<double>(ctx, P, K, L, atoms, weights, bary, s);
    return barycenter_t<float>(ctx, P, K, L, atoms, weights, bary, s);
  });
}

// evaluate_both (cpp/inverseWasserstein.h:986-1145) on device.  The gradient_both
// call allocates the arena first; the FP64 staging of this function lives in a
// second, small allocation owned by the context's arena tail.
int evaluate_both_dev(wdl_ctx* ctx, int P, int K, int L, int loss_type, double scale_dic,
                      const double* x, double* g, int n, const double* observed, double* f,
                      const double* b_storage, double* b_last, double* bary, cudaStream_t s) {
  const size_t N = ctx->N, KN = (size_t)K * N, PK = (size_t)P * K;
  if ((size_t)n != PK + KN) return set_error(ctx, WDL_ERR_INVALID_ARG, "n != P*K + K*N");
  // Staging: v2 weights [PK], v2 atoms [KN], la [PK], dic [KN], loss [P].
  const size_t stage = 8 * (2 * PK + 2 * KN + P) + 5 * 256;
  const size_t main = eval_bytes(ctx, P, K, L);
  int rc;
  if ((rc = ensure_arena(ctx, main + stage))) return rc;
  char* tail = static_cast<char*>(ctx->arena.ptr) + main;
  auto carve = [&](size_t nd) {
    double* p = reinterpret_cast<double*>(tail);
    tail += ((nd * 8 + 255) / 256) * 256;
    return p;
  };
  double* w2 = carve(PK);
  double* a2 = carve(KN);
  double* la = carve(PK);
  double* dic = carve(KN);
  double* loss = carve(P);
  // Back to the original domain and normalise (:997-1031).
  k_normalise_rows<<<P, 32, 0, s>>>(x, w2, K, scale_dic);
  WDL_LAUNCH_CHECK(ctx);
  k_normalise_rows<<<K, 256, 0, s>>>(x + PK, a2, N, 1.0);
  WDL_LAUNCH_CHECK(ctx);
  if ((rc = gradient_both_dev(ctx, P, K, L, loss_type, a2, w2, observed, b_storage, la, dic, bary,
                              loss, b_last, s, true)))
    return rc;
  k_project_weights<<<grid_for(P, 128, ctx->sm_count), 128, 0, s>>>(la, w2, g, P, K, scale_dic);
  WDL_LAUNCH_CHECK(ctx);
  k_project_atoms<<<K, 256, 0, s>>>(dic, a2, g + PK, N);
  WDL_LAUNCH_CHECK(ctx);
  k_sum_losses<<<1, 32, 0, s>>>(loss, f, P);
  WDL_LAUNCH_CHECK(ctx);
  return WDL_OK;
}

}  // namespace wdl
