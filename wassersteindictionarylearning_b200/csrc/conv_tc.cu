// Tensor-core (tcgen05) form of the separable Gaussian operator, and the FP32
// operator dispatch.
//
// For an image U (H x W, x fastest) the operator is out = G_H U G_W with the
// dense symmetric Gibbs factors (cpp/kernels.h:669-699).  One CTA computes a
// whole image with two tcgen05 GEMMs (M = 128 lanes = the x coordinate j):
//   MMA1: D1[j][i] = sum_k G[j][k] U[i][k]   (A = G, B = U; both K-major in SMEM)
//   MMA2: D2[j][i] = sum_m D1[j][m] G[i][m]  (A = D1 restaged to SMEM, B = G)
// so D2[j][i] = out[i][j].  D1 goes TMEM -> registers -> SMEM (as the next
// GEMM's K-major A operand) without leaving the SM, and D2 is read back with
// tcgen05.ld in which a warp's 32 lanes are 32 consecutive x: every global
// store of the epilogue is a coalesced 128-byte row segment.
//
// Precision: kind::tf32 (operands rounded to TF32, FP32 accumulate) or split
// BF16 (x = hi + lo, both BF16; hi*hi + hi*lo + lo*hi accumulated in FP32 with
// kind::f16), the latter ~2^-16 relative per product.
//
// Shared memory holds the factor G (resident for the CTA's lifetime) and one
// operand tile that is reused for U and for the restaged D1: 128 KB.  Operand
// tiles use the canonical 128-byte-swizzled K-major layout: a tile of 128 rows
// is split along K into 128-byte column blocks ("regions") of 128 x 128 B; in a
// region, row r's 16-byte chunk c sits at chunk position c ^ (r % 8).
#include <cuda_bf16.h>

#include "tc_ptx.cuh"
#include "wdl_internal.cuh"

namespace wdl {

struct TcResources {
  int max_side = 128;
  size_t smem_bytes = 0;
  int* d_err = nullptr;  // device status word written on a bounded-wait timeout
};

namespace {

constexpr int kRows = 128;               // tile rows (TMEM lanes / max grid side)
constexpr int kRegionBytes = kRows * 128; // one 128-byte column block of a tile
constexpr uint32_t kTmemCols = 256;      // D1: columns [0,128), D2: [128,256)
constexpr uint64_t kWaitNs = 2000000000ull;  // 2 s bound on every mbarrier wait
constexpr size_t kTileBytes = 64 * 1024;     // one operand (both planes)

template <bool SPLIT>
struct Fmt {
  static constexpr int esz = SPLIT ? 2 : 4;            // bytes per element
  static constexpr int kstep = SPLIT ? 16 : 8;          // K per MMA instruction
  static constexpr int plane_bytes = kRows * 128 * esz; // 32 KB (bf16) / 64 KB (tf32)
  static constexpr uint32_t fmt = SPLIT ? 1u : 2u;
};

__device__ __forceinline__ uint32_t swz(int r, int k, int esz) {
  const int per = 128 / esz;
  const int region = k / per;
  const int byte = (k - region * per) * esz;
  const int chunk = (byte >> 4) ^ (r & 7);
  return (uint32_t)(region * kRegionBytes + r * 128 + (chunk << 4) + (byte & 15));
}

__device__ __forceinline__ uint32_t to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

// Store one value at (r, k) of an operand tile (one or two planes).
template <bool SPLIT>
__device__ __forceinline__ void put1(uint8_t* tile, int r, int k, float v) {
  if (SPLIT) {
    const __nv_bfloat16 hi = __float2bfloat16_rn(v);
    const __nv_bfloat16 lo = __float2bfloat16_rn(v - __bfloat162float(hi));
    const uint32_t o = swz(r, k, 2);
    *reinterpret_cast<__nv_bfloat16*>(tile + o) = hi;
    *reinterpret_cast<__nv_bfloat16*>(tile + Fmt<true>::plane_bytes + o) = lo;
  } else {
    *reinterpret_cast<uint32_t*>(tile + swz(r, k, 4)) = to_tf32(v);
  }
}

// Store 16 consecutive K values (k0 % 16 == 0) of row r: whole 16-byte chunks.
template <bool SPLIT>
__device__ __forceinline__ void put16(uint8_t* tile, int r, int k0, const float (&v)[16]) {
  if (SPLIT) {
    uint32_t hi[8], lo[8];
#pragma unroll
    for (int t = 0; t < 8; ++t) {
      const __nv_bfloat162 h = __floats2bfloat162_rn(v[2 * t], v[2 * t + 1]);
      const float2 hf = __bfloat1622float2(h);
      const __nv_bfloat162 l = __floats2bfloat162_rn(v[2 * t] - hf.x, v[2 * t + 1] - hf.y);
      hi[t] = *reinterpret_cast<const uint32_t*>(&h);
      lo[t] = *reinterpret_cast<const uint32_t*>(&l);
    }
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      const uint32_t o = swz(r, k0 + 8 * c, 2);
      *reinterpret_cast<uint4*>(tile + o) = make_uint4(hi[4 * c], hi[4 * c + 1], hi[4 * c + 2], hi[4 * c + 3]);
      *reinterpret_cast<uint4*>(tile + Fmt<true>::plane_bytes + o) =
          make_uint4(lo[4 * c], lo[4 * c + 1], lo[4 * c + 2], lo[4 * c + 3]);
    }
  } else {
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const uint32_t o = swz(r, k0 + 4 * c, 4);
      *reinterpret_cast<uint4*>(tile + o) = make_uint4(to_tf32(v[4 * c]), to_tf32(v[4 * c + 1]),
                                                       to_tf32(v[4 * c + 2]), to_tf32(v[4 * c + 3]));
    }
  }
}

// D[128 x N] (+)= A[128 x K] * B[N x K]^T, A and B K-major tiles in SMEM.
template <bool SPLIT>
__device__ __forceinline__ void issue_gemm(uint32_t d_tmem, uint32_t a_tile, uint32_t b_tile,
                                           int K, int N) {
  using F = Fmt<SPLIT>;
  const uint32_t id = ptx::idesc(F::fmt, 128, (uint32_t)N);
  const int steps = K / F::kstep;
  for (int ks = 0; ks < steps; ++ks) {
    const uint32_t byte = (uint32_t)ks * 32u;
    const uint32_t off = (byte >> 7) * kRegionBytes + (byte & 127u);
    const uint64_t a = ptx::sw128_desc(a_tile + off);
    const uint64_t b = ptx::sw128_desc(b_tile + off);
    if (SPLIT) {
      const uint64_t alo = ptx::sw128_desc(a_tile + F::plane_bytes + off);
      const uint64_t blo = ptx::sw128_desc(b_tile + F::plane_bytes + off);
      ptx::mma_bf16(d_tmem, a, b, id, ks > 0 ? 1u : 0u);
      ptx::mma_bf16(d_tmem, a, blo, id, 1u);
      ptx::mma_bf16(d_tmem, alo, b, id, 1u);
    } else {
      ptx::mma_tf32(d_tmem, a, b, id, ks > 0 ? 1u : 0u);
    }
  }
}

// One image per loop iteration; grid-stride over the batch.  128 threads: warp w
// owns TMEM lanes 32w..32w+31 (x = 32w + lane).
template <bool SPLIT>
__global__ void __launch_bounds__(128, 1)
    tc_conv2d_kernel(const float* __restrict__ in, float* __restrict__ out, long long nimg, int W,
                     int H, int Wp, int Hp, const float* __restrict__ G, int Gn, int* err) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* base = reinterpret_cast<uint8_t*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint8_t* g_tile = base;
  uint8_t* x_tile = base + kTileBytes;
  uint64_t* bar = reinterpret_cast<uint64_t*>(base + 2 * kTileBytes);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(base + 2 * kTileBytes + 8);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t bar_a = ptx::smem_addr(bar);
  const uint32_t g_a = ptx::smem_addr(g_tile), x_a = ptx::smem_addr(x_tile);

  // Resident factor tile: G[r][k] = g(|r-k|) for r, k < Gn, zero elsewhere.
  for (int e = tid; e < kRows * kRows; e += blockDim.x) {
    const int r = e >> 7, k = e & 127;
    const float v = (r < Gn && k < Gn) ? G[(size_t)r * Gn + k] : 0.f;
    put1<SPLIT>(g_tile, r, k, v);
  }
  if (tid == 0) {
    ptx::mbar_init(bar_a, 1);
    ptx::fence_mbar_init();
  }
  if (warp == 0) ptx::tmem_alloc(ptx::smem_addr(tmem_slot), kTmemCols);
  ptx::fence_proxy_async_smem();
  ptx::tc_fence_before();
  __syncthreads();
  ptx::tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const uint32_t d1 = tmem, d2 = tmem + 128;
  const uint32_t lane_base = (uint32_t)(warp * 32) << 16;
  const int j = warp * 32 + lane;  // x coordinate owned by this thread
  uint32_t phase = 0;
  bool ok = true;

  for (long long img = blockIdx.x; img < nimg && ok; img += gridDim.x) {
    const float* src = in + (size_t)img * W * H;
    float* dst = out + (size_t)img * W * H;
    // U into the operand tile, zero-padded to Hp x Wp.
    for (int e = tid; e < Hp * Wp; e += blockDim.x) {
      const int i = e / Wp, k = e - i * Wp;
      const float v = (i < H && k < W) ? src[(size_t)i * W + k] : 0.f;
      put1<SPLIT>(x_tile, i, k, v);
    }
    ptx::fence_proxy_async_smem();
    __syncthreads();
    if (tid == 0) {
      ptx::tc_fence_after();
      issue_gemm<SPLIT>(d1, g_a, x_a, Wp, Hp);
      ptx::mma_commit(bar_a);
    }
    ok = __syncthreads_and(ptx::mbar_wait(bar_a, phase, kWaitNs)) != 0;
    phase ^= 1;
    ptx::tc_fence_after();
    // D1 -> SMEM as the K-major A operand of the second GEMM (row j, K = i).
    for (int c0 = 0; c0 < Hp; c0 += 16) {
      float v[16];
      ptx::tmem_ld16(d1 + lane_base + (uint32_t)c0, v);
      ptx::tmem_ld_wait();
      put16<SPLIT>(x_tile, j, c0, v);
    }
    ptx::tc_fence_before();
    ptx::fence_proxy_async_smem();
    __syncthreads();
    if (tid == 0) {
      ptx::tc_fence_after();
      issue_gemm<SPLIT>(d2, x_a, g_a, Hp, Hp);
      ptx::mma_commit(bar_a);
    }
    ok = __syncthreads_and(ok && ptx::mbar_wait(bar_a, phase, kWaitNs)) != 0;
    phase ^= 1;
    ptx::tc_fence_after();
    for (int c0 = 0; c0 < Hp; c0 += 16) {
      float v[16];
      ptx::tmem_ld16(d2 + lane_base + (uint32_t)c0, v);
      ptx::tmem_ld_wait();
      if (j < W) {
#pragma unroll
        for (int t = 0; t < 16; ++t)
          if (c0 + t < H) dst[(size_t)(c0 + t) * W + j] = v[t];
      }
    }
    ptx::tc_fence_before();
    __syncthreads();
  }
  if (!ok && tid == 0) atomicExch(err, WDL_ERR_TIMEOUT);
  __syncthreads();
  ptx::tc_fence_after();
  if (warp == 0) ptx::tmem_dealloc(tmem, kTmemCols);
}

}  // namespace

bool tc_supported(const wdl_ctx* ctx) {
  return ctx->ndim == 2 && ctx->W <= kRows && ctx->H <= kRows;
}

int tc_init(wdl_ctx* ctx) {
  if (!tc_supported(ctx))
    return set_error(ctx, WDL_ERR_UNSUPPORTED, "tensor-core operator needs a 2-D grid with sides <= 128");
  auto* r = new TcResources();
  r->smem_bytes = 2 * kTileBytes + 1024 + 64;
  ctx->tc = r;
  WDL_CUDA_TRY(ctx, cudaMalloc(&r->d_err, sizeof(int)));
  WDL_CUDA_TRY(ctx, cudaMemset(r->d_err, 0, sizeof(int)));
  WDL_CUDA_TRY(ctx, cudaFuncSetAttribute(tc_conv2d_kernel<true>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)r->smem_bytes));
  WDL_CUDA_TRY(ctx, cudaFuncSetAttribute(tc_conv2d_kernel<false>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)r->smem_bytes));
  return WDL_OK;
}

void tc_free(wdl_ctx* ctx) {
  if (!ctx->tc) return;
  if (ctx->tc->d_err) cudaFree(ctx->tc->d_err);
  delete ctx->tc;
  ctx->tc = nullptr;
}

static int conv_stack_tc(wdl_ctx* ctx, const float* in, float* out, size_t nimg, cudaStream_t s) {
  const int W = ctx->W, H = ctx->H;
  const int Wp = (W + 15) & ~15, Hp = (H + 15) & ~15;
  const int Gn = W >= H ? W : H;
  const float* G = ctx->G32[W >= H ? 0 : 1];
  const unsigned grid = (unsigned)(nimg < (size_t)ctx->sm_count ? nimg : (size_t)ctx->sm_count);
  if (ctx->precision == WDL_SPLIT_BF16)
    tc_conv2d_kernel<true><<<grid, 128, ctx->tc->smem_bytes, s>>>(in, out, (long long)nimg, W, H, Wp,
                                                                  Hp, G, Gn, ctx->tc->d_err);
  else
    tc_conv2d_kernel<false><<<grid, 128, ctx->tc->smem_bytes, s>>>(in, out, (long long)nimg, W, H, Wp,
                                                                   Hp, G, Gn, ctx->tc->d_err);
  WDL_LAUNCH_CHECK(ctx);
  return WDL_OK;
}

int conv_stack_f32(wdl_ctx* ctx, const float* in, float* out, float* tmp, size_t nimg,
                   cudaStream_t s) {
  if (nimg == 0) return WDL_OK;
  if (ctx->precision == WDL_FP32) return conv_stack_simt_f32(ctx, in, out, tmp, nimg, s);
  if (!ctx->tc) return set_error(ctx, WDL_ERR_UNSUPPORTED, "tensor-core operator not initialised");
  if (ctx->profiling) cudaEventRecord(ctx->ev_a, s);
  int rc = conv_stack_tc(ctx, in, out, nimg, s);
  if (rc) return rc;
  if (ctx->profiling) {
    cudaEventRecord(ctx->ev_b, s);
    cudaEventSynchronize(ctx->ev_b);
    float ms = 0;
    cudaEventElapsedTime(&ms, ctx->ev_a, ctx->ev_b);
    ctx->conv_ms += ms;
    ctx->conv_launches += 1;
    ctx->conv_images += (double)nimg;
  }
  return WDL_OK;
}

// Reads and clears the device status word of the tensor-core kernels.
int tc_check_status(wdl_ctx* ctx) {
  if (!ctx->tc) return WDL_OK;
  int h = 0;
  WDL_CUDA_TRY(ctx, cudaMemcpy(&h, ctx->tc->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (h != 0) {
    cudaMemset(ctx->tc->d_err, 0, sizeof(int));
    return set_error(ctx, h, "tensor-core kernel: a bounded wait timed out");
  }
  return WDL_OK;
}

}  // namespace wdl
