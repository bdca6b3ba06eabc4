// CUDA-core forms of the separable Gaussian operator (plain FP32 and FP64) and
// of the stabilised log-sum-exp operator.
//
// The reference applies the 2-D Gaussian as an x-pass into a transposed
// temporary followed by a y-pass (cpp/kernels.h:669-699) and the 3-D one as
// three such passes (:762-807).  Here every pass is the same primitive: an
// image viewed as [R][C] (C contiguous) is contracted along C with the dense
// C x C factor and written as [C][R], moving the contracted axis to the front.
// Applying it once per axis returns the image to its original layout.
#include "wdl_internal.cuh"

namespace wdl {
namespace {

// ---- dense axis pass: out[c][r] = sum_k in[r][k] * G[k][c] ----------------------
// Block tile 64 (r) x 64 (c), k-slab 16, 256 threads with a 4x4 register tile.
// Shared memory holds the input slab transposed (k-major) so both operands are
// read as contiguous 4-vectors.
constexpr int TR = 64, TC = 64, TK = 16;

template <typename T>
__global__ void __launch_bounds__(256) axis_pass_kernel(const T* __restrict__ in,
                                                        T* __restrict__ out,
                                                        const T* __restrict__ G, int R, int C,
                                                        size_t img_stride) {
  __shared__ __align__(16) T sA[TK][TR + 4];
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
      for (int i = 0; i < 4; ++i) a[i] = sA[kk][tr * 4 + i];
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
      int r = r0 + tr * 4 + i;
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
// A block owns LR rows of one image and produces every output of those rows.
constexpr int LR = 16;

template <typename T>
__device__ __forceinline__ T dev_exp(T x);
template <>
__device__ __forceinline__ float dev_exp<float>(float x) { return expf(x); }
template <>
__device__ __forceinline__ double dev_exp<double>(double x) { return exp(x); }
template <typename T>
__device__ __forceinline__ T dev_log(T x);
template <>
__device__ __forceinline__ float dev_log<float>(float x) { return logf(x); }
template <>
__device__ __forceinline__ double dev_log<double>(double x) { return log(x); }

template <typename T, bool SIGNED>
__global__ void __launch_bounds__(256) log_axis_pass_kernel(
    const T* __restrict__ in, T* __restrict__ out, int R, int C, size_t img_stride, T gamma_t,
    const uint8_t* __restrict__ in_sign, uint8_t* __restrict__ out_sign) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* rows = reinterpret_cast<T*>(smem_raw);           // [LR][C]
  T* lk = rows + LR * C;                                // [C] : -d^2/gamma
  uint8_t* sg = reinterpret_cast<uint8_t*>(lk + C);     // [LR][C]
  const int r0 = blockIdx.x * LR;
  const size_t base = (size_t)blockIdx.y * img_stride;
  const int nr = min(LR, R - r0);
  for (int e = threadIdx.x; e < LR * C; e += blockDim.x) {
    int rr = e / C, k = e - rr * C;
    T v = T(0);
    uint8_t sv = 1;
    if (rr < nr) {
      v = in[base + (size_t)(r0 + rr) * C + k];
      if (SIGNED) sv = in_sign[base + (size_t)(r0 + rr) * C + k];
    }
    rows[e] = v;
    if (SIGNED) sg[e] = sv;
  }
  for (int d = threadIdx.x; d < C; d += blockDim.x) lk[d] = -T(d * d) / gamma_t;
  __syncthreads();
  // Thread -> (c, rr) with rr fastest so that stores out[c][r0+rr] are contiguous.
  for (int e = threadIdx.x; e < LR * C; e += blockDim.x) {
    int c = e / LR, rr = e - c * LR;
    if (rr >= nr) continue;
    const T* row = rows + rr * C;
    // The reference starts the maximum at -1e99 (FP64); FP32 uses -FLT_MAX so that
    // an all -inf row still sums to 0 and returns -inf instead of NaN.
    T vmax = sizeof(T) == 8 ? T(-1e99) : T(-3.402823466e38);
    for (int k = 0; k < C; ++k) {
      T t = lk[abs(c - k)] + row[k];
      vmax = t > vmax ? t : vmax;
    }
    T sum = T(0);
    for (int k = 0; k < C; ++k) {
      T ex = dev_exp<T>(lk[abs(c - k)] + row[k] - vmax);
      if (SIGNED) sum += sg[rr * C + k] ? ex : -ex;
      else sum += ex;
    }
    size_t o = base + (size_t)c * R + (r0 + rr);
    if (SIGNED) {
      out_sign[o] = sum >= T(0) ? 1 : 0;
      out[o] = dev_log<T>(fabs(sum)) + vmax;
    } else {
      out[o] = dev_log<T>(sum) + vmax;
    }
  }
}

template <typename T>
int log_axis_pass(wdl_ctx* ctx, const T* in, T* out, int R, int C, size_t nimg, size_t img_stride,
                  const uint8_t* in_sign, uint8_t* out_sign, cudaStream_t s) {
  size_t smem = (size_t)LR * C * sizeof(T) + C * sizeof(T) + (size_t)LR * C + 16;
  const T gamma_t = T(ctx->gamma);
  size_t done = 0;
  while (done < nimg) {
    size_t chunk = nimg - done;
    if (chunk > 65535) chunk = 65535;
    dim3 grid((R + LR - 1) / LR, (unsigned)chunk);
    size_t off = done * img_stride;
    if (in_sign) {
      auto k = log_axis_pass_kernel<T, true>;
      if (smem > 48 * 1024) cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      k<<<grid, 256, smem, s>>>(in + off, out + off, R, C, img_stride, gamma_t, in_sign + off,
                                out_sign + off);
    } else {
      auto k = log_axis_pass_kernel<T, false>;
      if (smem > 48 * 1024) cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      k<<<grid, 256, smem, s>>>(in + off, out + off, R, C, img_stride, gamma_t, nullptr, nullptr);
    }
    WDL_LAUNCH_CHECK(ctx);
    done += chunk;
  }
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
  ConvTimer(wdl_ctx* c, cudaStream_t st, size_t n) : ctx(c), s(st), nimg(n) {
    if (ctx->profiling) cudaEventRecord(ctx->ev_a, s);
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
  ConvTimer timer(ctx, s, nimg);
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
