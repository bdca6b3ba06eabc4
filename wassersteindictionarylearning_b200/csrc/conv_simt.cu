// CUDA-core forms of the separable Gaussian operator (plain FP32 and FP64) and
// of the stabilised log-sum-exp operator.
//
// The reference applies the 2-D Gaussian as an x-pass into a transposed
// temporary followed by a y-pass (cpp/kernels.h:669-699) and the 3-D one as
// three such passes (:762-807).  Here every pass is the same primitive: an
// image viewed as [R][C] (C contiguous) is contracted along C with the dense
// C x C factor and written as [C][R], moving the contracted axis to the front.
// Applying it once per axis returns the image to its original layout.
#include <cstdlib>
#include <cstring>

#include "wdl_internal.cuh"

namespace wdl {
namespace {

// ---- dense axis pass: out[c][r] = sum_k in[r][k] * G[k][c] ----------------------
// Block tile 64 (r) x 64 (c), k-slab 16, 256 threads with a 4x4 register tile
// (thread (tr, tc) owns 4 rows and the columns 4 tc + j).  Shared memory holds
// the input slab transposed (k-major).  FP32: the thread's rows are 4 tr + i,
// read as one 16-byte vector per k (row stride TR + 4 keeps it aligned; a
// quarter-warp reads 128 contiguous bytes).  FP64: the rows are tr + 16 i,
// read as 4 scalars per k: the 16 tr of a warp read 16 consecutive doubles, one
// conflict-free wavefront, where 16-byte vectors of doubles 32 bytes apart
// would conflict two ways; row stride TR + 1 spreads the slab's stores over
// the banks.  The two tc of a warp read two broadcast 4-vectors of the factor.
constexpr int TR = 64, TC = 64, TK = 16;

template <typename T>
struct AxisRows {
  static constexpr bool kInterleaved = sizeof(T) == 8;
  static constexpr int kStride = kInterleaved ? TR + 1 : TR + 4;
  __device__ static int row(int tr, int i) { return kInterleaved ? tr + 16 * i : 4 * tr + i; }
};

template <typename T>
__global__ void __launch_bounds__(256) axis_pass_kernel(const T* __restrict__ in,
                                                        T* __restrict__ out,
                                                        const T* __restrict__ G, int R, int C,
                                                        size_t img_stride) {
  using Rw = AxisRows<T>;
  __shared__ __align__(16) T sA[TK][Rw::kStride];
  __shared__ __align__(16) T sB[TK][TC + 4];
  const int tid = threadIdx.x;
  const int tr = tid & 15, tc = tid >> 4;
  const int r0 = blockIdx.x * TR, c0 = blockIdx.y * TC;
  const T* src = in + (size_t)blockIdx.z * img_stride;
  T* dst = out + (size_t)blockIdx.z * img_stride;

  T acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = T(0);

  for (int k0 = 0; k0 < C; k0 += TK) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      int e = tid + 256 * q;
      int rr = e >> 4, kk = e & 15;
      int r = r0 + rr, k = k0 + kk;
      sA[kk][rr] = (r < R && k < C) ? src[(size_t)r * C + k] : T(0);
      int kb = e >> 6, cc = e & 63;
      int kg = k0 + kb, c = c0 + cc;
      sB[kb][cc] = (kg < C && c < C) ? G[(size_t)kg * C + c] : T(0);
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < TK; ++kk) {
      T a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = sA[kk][Rw::row(tr, i)];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = sB[kk][tc * 4 + j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    int c = c0 + tc * 4 + j;
    if (c >= C) continue;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      int r = r0 + Rw::row(tr, i);
      if (r < R) dst[(size_t)c * R + r] = acc[i][j];
    }
  }
}

template <typename T>
int axis_pass(wdl_ctx* ctx, const T* in, T* out, const T* G, int R, int C, size_t nimg,
              size_t img_stride, cudaStream_t s) {
  size_t done = 0;
  while (done < nimg) {  // gridDim.z is limited to 65535
    size_t chunk = nimg - done;
    if (chunk > 65535) chunk = 65535;
    dim3 grid((R + TR - 1) / TR, (C + TC - 1) / TC, (unsigned)chunk);
    axis_pass_kernel<T><<<grid, 256, 0, s>>>(in + done * img_stride, out + done * img_stride, G,
                                             R, C, img_stride);
    WDL_LAUNCH_CHECK(ctx);
    done += chunk;
  }
  return WDL_OK;
}

// ---- log-domain axis pass ---------------------------------------------------------
// out[c][r] = log sum_k s_k exp(-(c-k)^2/gamma + in[r][k]) with the reference's
// two passes per output: the maximum of the exponents, then the shifted sum
// (cpp/kernels.h:1082-1091).  With signs, s_k = +-1 from in_sign and the sign of
// the sum goes to out_sign, log|sum| to out (cpp/kernels.h:1123-1136).
//
// A block owns LR rows of one image (staged in SMEM with an odd row stride, so
// the rows a warp reads at one tap fall in different banks) and produces every
// output of those rows.  Taps are visited outwards from k = c, both sides per
// step.  With X = max_k in[r][k], every tap at distance >= d has exponent
// <= -d^2/gamma + X, so:
//  * the maximum pass stops at the first d where -d^2/gamma + X <= max so far;
//  * the sum pass stops at the first d where -d^2/gamma + X < max - kTail; the
//    taps left out add at most 2C e^-kTail relative to the largest term, below
//    the rounding of the sum (kTail = 40 bits for FP32, 60 nats for FP64), so
//    the result is the full sum's to rounding.
// FP32 works in base 2 (inputs scaled by log2 e once when staged; ex2 / lg2),
// FP64 in base e with exp / log.  The summation order (outwards, both sides)
// differs from the reference's k = 0..C-1; only rounding depends on it.  LR
// (rows per block) is chosen per shape by the autotuner below; every output is
// computed by the same operations whatever LR is, so the choice never changes
// a result.
constexpr int kLogRowsDefault = 16;

template <typename T>
struct LogOps;
template <>
struct LogOps<float> {
  static constexpr float kScale = 1.4426950408889634f;   // log2 e: natural -> base 2
  static constexpr float kUnscale = 0.6931471805599453f;  // ln 2
  static constexpr float kTail = 40.f;                   // bits
  static constexpr float kFloor = -3.402823466e38f;      // start of the maximum
  // the hardware base-2 exponential; arguments are <= 0 here and results
  // below 2^-126 are far under the sum's rounding, so flushing them is exact
  __device__ static float ex(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
  }
  // the hardware base-2 logarithm: absolute error ~2^-22 on log2, below the
  // FP32 rounding of the result (lg + max) * ln 2 once |result| > 1
  __device__ static float lg(float x) {
    float y;
    asm("lg2.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
  }
};
template <>
struct LogOps<double> {
  static constexpr double kScale = 1.0;
  static constexpr double kUnscale = 1.0;
  static constexpr double kTail = 60.0;   // nats
  static constexpr double kFloor = -1e99;  // the reference's start (cpp/kernels.h:1083)
  __device__ static double ex(double x) { return exp(x); }
  __device__ static double lg(double x) { return log(x); }
};

// One output of the log-domain pass: out = log |sum_k s_k exp(lk[|c-k|] + row[k])|
// (in the kernel's base) and its sign, by the two passes described above.  Both
// kernel layouts below call this, so an output's arithmetic does not depend on
// the layout.  *taps receives the number of exponentials evaluated.
template <typename T, bool SIGNED>
__device__ __forceinline__ T log_out(const T* __restrict__ row, const uint8_t* __restrict__ sgn,
                                     const T* __restrict__ lk, T X, int c, int C, bool* pos, unsigned* taps) {
  using Op = LogOps<T>;
  const int dboth = min(c, C - 1 - c);      // both sides inside the row for d <= dboth
  const int sgnd = c < C - 1 - c ? 1 : -1;  // the side that remains beyond dboth
  T m = row[c] > Op::kFloor ? row[c] : Op::kFloor;
  int d = 1;
  for (; d <= dboth; ++d) {
    const T l = lk[d];
    if (l + X <= m) break;
    const T a = l + row[c - d], b = l + row[c + d];
    const T ab = a > b ? a : b;
    m = ab > m ? ab : m;
  }
  if (d > dboth) {
    for (; d < C && (sgnd > 0 ? c + d < C : c - d >= 0); ++d) {
      const T l = lk[d];
      if (l + X <= m) break;
      const T t = l + row[c + sgnd * d];
      m = t > m ? t : m;
    }
  }
  T sum = Op::ex(row[c] - m);
  if (SIGNED && !sgn[c]) sum = -sum;
  const T fl = m - Op::kTail;
  for (d = 1; d <= dboth; ++d) {
    const T l = lk[d];
    if (l + X < fl) break;
    const T lm = l - m;
    const T ea = Op::ex(lm + row[c - d]), eb = Op::ex(lm + row[c + d]);
    if (SIGNED) sum += (sgn[c - d] ? ea : -ea) + (sgn[c + d] ? eb : -eb);
    else sum += ea + eb;
  }
  if (d > dboth) {
    for (; d < C && (sgnd > 0 ? c + d < C : c - d >= 0); ++d) {
      const T l = lk[d];
      if (l + X < fl) break;
      const int k = c + sgnd * d;
      const T ex = Op::ex((l - m) + row[k]);
      sum += (!SIGNED || sgn[k]) ? ex : -ex;
    }
  }
  const int dmax = d - 1;  // the last tap distance summed
  *taps += 1 + min(dmax, c) + min(dmax, C - 1 - c);
  if (SIGNED) {
    *pos = sum >= T(0);
    return (Op::lg(fabs(sum)) + m) * Op::kUnscale;
  }
  *pos = true;
  return (Op::lg(sum) + m) * Op::kUnscale;
}

// Stage LR rows of one image in SMEM (odd row stride CP), their signs, the row
// maxima X and the tap table lk[d] = -d^2/gamma (scaled).
template <typename T, bool SIGNED, int LR>
__device__ __forceinline__ void log_stage(const T* __restrict__ in, const uint8_t* __restrict__ in_sign,
                                          T* rows, uint8_t* sg, T* xmax, T* lk, size_t base, int r0, int nr,
                                          int C, int CP, int SP, T gamma_t) {
  using Op = LogOps<T>;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // warp w owns rows w, w + 8, ..., so the row maxima come from shuffles
  for (int rr = warp; rr < LR; rr += 8) {
    T vm = Op::kFloor;
    for (int k = lane; k < C; k += 32) {
      T v = Op::kFloor;
      uint8_t sv = 1;
      if (rr < nr) {
        v = in[base + (size_t)(r0 + rr) * C + k] * Op::kScale;
        if (SIGNED) sv = in_sign[base + (size_t)(r0 + rr) * C + k];
      }
      rows[rr * CP + k] = v;
      if (SIGNED) sg[rr * SP + k] = sv;
      vm = v > vm ? v : vm;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const T w = __shfl_xor_sync(0xffffffffu, vm, o);
      vm = w > vm ? w : vm;
    }
    if (lane == 0) xmax[rr] = vm;
  }
  for (int d = threadIdx.x; d < C; d += blockDim.x) lk[d] = -T(d) * T(d) / gamma_t * Op::kScale;
}

// Layout "rows fastest": a block owns LR rows of one image and thread e makes
// output (c = e / LR, rr = e % LR), so the stores out[c][r0 + rr] of a warp are
// contiguous runs.
template <typename T, bool SIGNED, int LR>
__global__ void __launch_bounds__(256) log_axis_pass_kernel(
    const T* __restrict__ in, T* __restrict__ out, int R, int C, size_t img_stride, T gamma_t,
    const uint8_t* __restrict__ in_sign, uint8_t* __restrict__ out_sign,
    unsigned long long* __restrict__ exps) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int CP = C + 1;                                 // odd row stride (elements)
  T* rows = reinterpret_cast<T*>(smem_raw);             // [LR][CP]
  T* lk = rows + LR * CP;                               // [C]: -d^2/gamma (scaled)
  T* xmax = lk + C;                                     // [LR]
  uint8_t* sg = reinterpret_cast<uint8_t*>(xmax + LR);  // [LR][C + 4] (bank-spread bytes)
  const int SP = C + 4;
  const int r0 = blockIdx.x * LR;
  const size_t base = (size_t)blockIdx.y * img_stride;
  const int nr = min(LR, R - r0);
  const int lane = threadIdx.x & 31;
  log_stage<T, SIGNED, LR>(in, in_sign, rows, sg, xmax, lk, base, r0, nr, C, CP, SP, gamma_t);
  __syncthreads();
  unsigned n_ex = 0;  // exps evaluated by this thread (profiling only)
  for (int e = threadIdx.x; e < LR * C; e += blockDim.x) {
    const int c = e / LR, rr = e - c * LR;
    if (rr >= nr) continue;
    bool pos;
    const T v = log_out<T, SIGNED>(rows + rr * CP, sg + rr * SP, lk, xmax[rr], c, C, &pos, &n_ex);
    const size_t o = base + (size_t)c * R + (r0 + rr);
    out[o] = v;
    if (SIGNED) out_sign[o] = pos ? 1 : 0;
  }
  if (exps) {
    unsigned long long v = n_ex;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) atomicAdd(exps, v);
  }
}

// Layout "row per warp": warp w makes the outputs of rows w, w + 8, ..., its
// lanes taking 32 consecutive c of one row, so the lanes of a warp run nearly
// the same number of taps (neighbouring outputs of one row) and read
// consecutive SMEM words; the results go through SMEM ([C][LR + 1]) and are
// stored as contiguous runs of out[c][r0..].  Same outputs, bit for bit, as
// the layout above.
template <typename T, bool SIGNED, int LR>
__global__ void __launch_bounds__(256) log_axis_pass_rowwarp_kernel(
    const T* __restrict__ in, T* __restrict__ out, int R, int C, size_t img_stride, T gamma_t,
    const uint8_t* __restrict__ in_sign, uint8_t* __restrict__ out_sign,
    unsigned long long* __restrict__ exps) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int CP = C + 1;
  T* rows = reinterpret_cast<T*>(smem_raw);             // [LR][CP]
  T* lk = rows + LR * CP;                               // [C]
  T* xmax = lk + C;                                     // [LR]
  T* ot = xmax + LR;                                    // [C][LR + 1] results
  uint8_t* sg = reinterpret_cast<uint8_t*>(ot + (size_t)C * (LR + 1));  // [LR][C + 4]
  const int SP = C + 4;
  uint8_t* osg = sg + LR * SP;                          // [C][LR + 1] result signs
  const int r0 = blockIdx.x * LR;
  const size_t base = (size_t)blockIdx.y * img_stride;
  const int nr = min(LR, R - r0);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  log_stage<T, SIGNED, LR>(in, in_sign, rows, sg, xmax, lk, base, r0, nr, C, CP, SP, gamma_t);
  __syncthreads();
  unsigned n_ex = 0;
  for (int rr = warp; rr < nr; rr += 8) {
    const T* row = rows + rr * CP;
    const uint8_t* sgn = sg + rr * SP;
    const T X = xmax[rr];
    for (int c = lane; c < C; c += 32) {
      bool pos;
      ot[(size_t)c * (LR + 1) + rr] = log_out<T, SIGNED>(row, sgn, lk, X, c, C, &pos, &n_ex);
      if (SIGNED) osg[(size_t)c * (LR + 1) + rr] = pos ? 1 : 0;
    }
  }
  __syncthreads();
  for (int e = threadIdx.x; e < LR * C; e += blockDim.x) {
    const int c = e / LR, rr = e - c * LR;
    if (rr >= nr) continue;
    const size_t o = base + (size_t)c * R + (r0 + rr);
    out[o] = ot[(size_t)c * (LR + 1) + rr];
    if (SIGNED) out_sign[o] = osg[(size_t)c * (LR + 1) + rr];
  }
  if (exps) {
    unsigned long long v = n_ex;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) atomicAdd(exps, v);
  }
}

template <typename T>
size_t log_axis_smem(int LR, int C, bool rowwarp = false) {
  size_t b = ((size_t)LR * (C + 1) + C + LR) * sizeof(T) + (size_t)LR * (C + 4) + 16;
  if (rowwarp) b += (size_t)C * (LR + 1) * (sizeof(T) + 1);
  return b;
}

template <typename T, int LR, bool ROWWARP>
int log_axis_launch(wdl_ctx* ctx, const T* in, T* out, int R, int C, size_t nimg, size_t img_stride,
                    const uint8_t* in_sign, uint8_t* out_sign, cudaStream_t s) {
  const size_t smem = log_axis_smem<T>(LR, C, ROWWARP);
  const T gamma_t = T(ctx->gamma);
  size_t done = 0;
  while (done < nimg) {
    size_t chunk = nimg - done;
    if (chunk > 65535) chunk = 65535;
    dim3 grid((R + LR - 1) / LR, (unsigned)chunk);
    size_t off = done * img_stride;
    if (in_sign) {
      auto k = ROWWARP ? log_axis_pass_rowwarp_kernel<T, true, LR> : log_axis_pass_kernel<T, true, LR>;
      if (smem > 48 * 1024) cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      k<<<grid, 256, smem, s>>>(in + off, out + off, R, C, img_stride, gamma_t, in_sign + off,
                                out_sign + off, ctx->profiling ? ctx->d_taps : nullptr);
    } else {
      auto k = ROWWARP ? log_axis_pass_rowwarp_kernel<T, false, LR> : log_axis_pass_kernel<T, false, LR>;
      if (smem > 48 * 1024) cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      k<<<grid, 256, smem, s>>>(in + off, out + off, R, C, img_stride, gamma_t, nullptr, nullptr,
                                ctx->profiling ? ctx->d_taps : nullptr);
    }
    WDL_LAUNCH_CHECK(ctx);
    done += chunk;
  }
  return WDL_OK;
}


template <typename T>
int log_axis_dispatch(wdl_ctx* ctx, int LR, const T* in, T* out, int R, int C, size_t nimg,
                      size_t img_stride, const uint8_t* in_sign, uint8_t* out_sign, cudaStream_t s) {
  // choice: rows per block (LR), plus 100 for the row-per-warp layout
  switch (LR) {
    case 8: return log_axis_launch<T, 8, false>(ctx, in, out, R, C, nimg, img_stride, in_sign, out_sign, s);
    case 32: return log_axis_launch<T, 32, false>(ctx, in, out, R, C, nimg, img_stride, in_sign, out_sign, s);
    case 108: return log_axis_launch<T, 8, true>(ctx, in, out, R, C, nimg, img_stride, in_sign, out_sign, s);
    case 116: return log_axis_launch<T, 16, true>(ctx, in, out, R, C, nimg, img_stride, in_sign, out_sign, s);
    case 132: return log_axis_launch<T, 32, true>(ctx, in, out, R, C, nimg, img_stride, in_sign, out_sign, s);
    default: return log_axis_launch<T, 16, false>(ctx, in, out, R, C, nimg, img_stride, in_sign, out_sign, s);
  }
}

// Autotuner: the first call of a shape (rows, row length, image count, type,
// signed) outside a graph capture runs every candidate rows-per-block on the
// call's own data (once untimed, once timed with CUDA events on the call's
// stream) and keeps the fastest for later calls of that shape.  WDL_AUTOTUNE=0
// keeps the default.
template <typename T>
int log_axis_pass(wdl_ctx* ctx, const T* in, T* out, int R, int C, size_t nimg, size_t img_stride,
                  const uint8_t* in_sign, uint8_t* out_sign, cudaStream_t s) {
  const long long key[6] = {1, R, C, (long long)nimg, (long long)sizeof(T), in_sign ? 1 : 0};
  for (const auto& e : ctx->tuned)
    if (!std::memcmp(e.key, key, sizeof(key)))
      return log_axis_dispatch<T>(ctx, e.choice, in, out, R, C, nimg, img_stride, in_sign, out_sign, s);
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  cudaStreamIsCapturing(s, &cap);
  if (!autotune_enabled() || !ctx->autotune || cap != cudaStreamCaptureStatusNone || ctx->profiling)
    return log_axis_dispatch<T>(ctx, kLogRowsDefault, in, out, R, C, nimg, img_stride, in_sign, out_sign, s);
  const int cand[6] = {8, 16, 32, 108, 116, 132};
  int best = kLogRowsDefault;
  float best_ms = 1e30f;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  WDL_CUDA_TRY(ctx, cudaEventCreate(&e0));
  WDL_CUDA_TRY(ctx, cudaEventCreate(&e1));
  int rc = WDL_OK;
  for (int c : cand) {
    if (log_axis_smem<T>(c % 100, C, c >= 100) > 200 * 1024) continue;
    // an untimed run first: the first launch of a variant also loads it
    if ((rc = log_axis_dispatch<T>(ctx, c, in, out, R, C, nimg, img_stride, in_sign, out_sign, s))) break;
    cudaEventRecord(e0, s);
    if ((rc = log_axis_dispatch<T>(ctx, c, in, out, R, C, nimg, img_stride, in_sign, out_sign, s))) break;
    cudaEventRecord(e1, s);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best_ms) {
      best_ms = ms;
      best = c;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  wdl_ctx::TuneEntry t;
  std::memcpy(t.key, key, sizeof(key));
  t.choice = best;
  t.ms = best_ms;
  ctx->tuned.push_back(t);
  // the candidates computed identical outputs; the last one's stands
  return WDL_OK;
}

template <typename T>
const T* factor(const wdl_ctx* ctx, int axis);
template <>
const float* factor<float>(const wdl_ctx* ctx, int axis) { return ctx->G32[axis]; }
template <>
const double* factor<double>(const wdl_ctx* ctx, int axis) { return ctx->G64[axis]; }

struct ConvTimer {
  wdl_ctx* ctx;
  cudaStream_t s;
  size_t nimg;
  bool count_exps;
  ConvTimer(wdl_ctx* c, cudaStream_t st, size_t n, bool exps = false)
      : ctx(c), s(st), nimg(n), count_exps(exps && c->profiling) {
    if (!ctx->profiling) return;
    if (count_exps) {
      if (!ctx->d_taps && cudaMalloc(&ctx->d_taps, sizeof(unsigned long long)) != cudaSuccess) {
        ctx->d_taps = nullptr;
        count_exps = false;
      }
      if (count_exps) cudaMemsetAsync(ctx->d_taps, 0, sizeof(unsigned long long), s);
    }
    cudaEventRecord(ctx->ev_a, s);
  }
  void done() {
    if (!ctx->profiling) return;
    cudaEventRecord(ctx->ev_b, s);
    cudaEventSynchronize(ctx->ev_b);
    float ms = 0;
    cudaEventElapsedTime(&ms, ctx->ev_a, ctx->ev_b);
    ctx->conv_ms += ms;
    ctx->conv_launches += 1;
    ctx->conv_images += (double)nimg;
    if (count_exps) {
      unsigned long long h = 0;
      if (cudaMemcpy(&h, ctx->d_taps, sizeof(h), cudaMemcpyDeviceToHost) == cudaSuccess)
        ctx->log_exps += (double)h;
    }
  }
};

template <typename T>
int conv_stack_simt(wdl_ctx* ctx, const T* in, T* out, T* tmp, size_t nimg, cudaStream_t s) {
  const int W = ctx->W, H = ctx->H, D = ctx->D;
  const size_t N = ctx->N;
  ConvTimer timer(ctx, s, nimg);
  int rc;
  if (ctx->ndim == 2) {
    if ((rc = axis_pass<T>(ctx, in, tmp, factor<T>(ctx, 0), H, W, nimg, N, s))) return rc;
    if ((rc = axis_pass<T>(ctx, tmp, out, factor<T>(ctx, 1), W, H, nimg, N, s))) return rc;
  } else {
    if ((rc = axis_pass<T>(ctx, in, out, factor<T>(ctx, 0), D * H, W, nimg, N, s))) return rc;
    if ((rc = axis_pass<T>(ctx, out, tmp, factor<T>(ctx, 1), W * D, H, nimg, N, s))) return rc;
    if ((rc = axis_pass<T>(ctx, tmp, out, factor<T>(ctx, 2), H * W, D, nimg, N, s))) return rc;
  }
  timer.done();
  return WDL_OK;
}

template <typename T>
int log_conv_stack_simt(wdl_ctx* ctx, const T* in, T* out, T* tmp, size_t nimg,
                        const uint8_t* in_sign, uint8_t* out_sign, uint8_t* tmp_sign,
                        cudaStream_t s) {
  if (ctx->ndim != 2)
    return set_error(ctx, WDL_ERR_UNSUPPORTED, "log-domain operator is 2-D only (as the reference)");
  const int W = ctx->W, H = ctx->H;
  const size_t N = ctx->N;
  ConvTimer timer(ctx, s, nimg, true);
  int rc;
  if ((rc = log_axis_pass<T>(ctx, in, tmp, H, W, nimg, N, in_sign, in_sign ? tmp_sign : nullptr, s)))
    return rc;
  if ((rc = log_axis_pass<T>(ctx, tmp, out, W, H, nimg, N, in_sign ? tmp_sign : nullptr, out_sign, s)))
    return rc;
  timer.done();
  return WDL_OK;
}

}  // namespace

int conv_stack_f64(wdl_ctx* ctx, const double* in, double* out, double* tmp, size_t nimg,
                   cudaStream_t s) {
  return conv_stack_simt<double>(ctx, in, out, tmp, nimg, s);
}

int conv_stack_simt_f32(wdl_ctx* ctx, const float* in, float* out, float* tmp, size_t nimg,
                        cudaStream_t s) {
  return conv_stack_simt<float>(ctx, in, out, tmp, nimg, s);
}

int log_conv_stack_f32(wdl_ctx* ctx, const float* in, float* out, float* tmp, size_t nimg,
                       const uint8_t* in_sign, uint8_t* out_sign, uint8_t* tmp_sign,
                       cudaStream_t s) {
  return log_conv_stack_simt<float>(ctx, in, out, tmp, nimg, in_sign, out_sign, tmp_sign, s);
}

int log_conv_stack_f64(wdl_ctx* ctx, const double* in, double* out, double* tmp, size_t nimg,
                       const uint8_t* in_sign, uint8_t* out_sign, uint8_t* tmp_sign,
                       cudaStream_t s) {
  return log_conv_stack_simt<double>(ctx, in, out, tmp, nimg, in_sign, out_sign, tmp_sign, s);
}

}  // namespace wdl
