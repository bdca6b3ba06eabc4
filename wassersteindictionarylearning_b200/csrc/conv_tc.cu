// Tensor-core (tcgen05) form of the separable Gaussian operator, and the FP32
// operator dispatch.
//
// For an image U (H x W, x fastest) the operator is out = G_H U G_W with the
// dense symmetric Gibbs factors (cpp/kernels.h:669-699).  One CTA computes a
// whole image with two tcgen05 GEMMs (M = 128 lanes = the x coordinate j):
//   MMA1: D1[j][i] = sum_k G[j][k] U[i][k]   (A = G, B = U; both K-major in SMEM)
//   MMA2: D2[j][i] = sum_m D1[j][m] G[i][m]  (A = D1 restaged in TMEM, B = G)
// so D2[j][i] = out[i][j].  D1 goes TMEM -> registers -> TMEM (split into
// BF16 hi / lo, or rounded to TF32) as the next GEMM's A operand, which
// tcgen05.mma reads from tensor memory, and D2 is read back with tcgen05.ld in
// which a warp's 32 lanes are 32 consecutive x: every global store of the
// epilogue is a coalesced 128-byte row segment.
//
// Precision: kind::tf32 (operands rounded to TF32, FP32 accumulate) or split
// BF16 (x = hi + lo, both BF16; hi*hi + hi*lo + lo*hi accumulated in FP32 with
// kind::f16), the latter ~2^-16 relative per product.
//
// Shared memory holds the factor G (resident for the CTA's lifetime) and one
// operand tile per warpgroup for U.  Operand
// tiles use the canonical 128-byte-swizzled K-major layout: a tile of 128 rows
// is split along K into 128-byte column blocks ("regions") of 128 x 128 B; in a
// region, row r's 16-byte chunk c sits at chunk position c ^ (r % 8).
#include "tc_common.cuh"

namespace wdl {

struct TcResources {
  bool fused = false;    // 2-D with sides <= 128: whole-image operator and fused Sinkhorn kernel
  uint8_t* factor_blocks[3] = {nullptr, nullptr, nullptr};  // axis-pass operand blocks per axis
  size_t smem_bytes = 0;
  int* d_err = nullptr;  // device status word written on a bounded-wait timeout
};

namespace {

using namespace tc;

// Image U (H x W fp32, row-major) -> operand tile rows i < Hp, K = k < Wp, zero
// padded.  Work unit: one 16-byte SMEM chunk of one row (8 BF16 or 4 TF32
// values); a thread issues the global loads of UNR chunks before converting any
// of them so that many loads are in flight.
template <bool SPLIT>
__device__ __forceinline__ void stage_image(uint8_t* tile, const float* __restrict__ src, int W,
                                            int H, int Wp, int Hp, int t, bool vec) {
  constexpr int CE = SPLIT ? 8 : 4;  // elements per chunk
  constexpr int UNR = 8;
  const int cpr = Wp / CE;           // chunks per row
  const int total = Hp * cpr;
  for (int base = t; base < total; base += 128 * UNR) {
    float v[UNR][CE];
#pragma unroll
    for (int u = 0; u < UNR; ++u) {
      const int c = base + u * 128;
      const int i = c / cpr, k0 = (c - i * cpr) * CE;
      if (c < total && i < H) {
        const float* row = src + (size_t)i * W;
        if (vec && k0 + CE <= W) {
#pragma unroll
          for (int q = 0; q < CE; q += 4) {
            const float4 f = __ldg(reinterpret_cast<const float4*>(row + k0 + q));
            v[u][q] = f.x; v[u][q + 1] = f.y; v[u][q + 2] = f.z; v[u][q + 3] = f.w;
          }
        } else {
#pragma unroll
          for (int q = 0; q < CE; ++q) v[u][q] = (k0 + q < W) ? __ldg(row + k0 + q) : 0.f;
        }
      } else {
#pragma unroll
        for (int q = 0; q < CE; ++q) v[u][q] = 0.f;
      }
    }
#pragma unroll
    for (int u = 0; u < UNR; ++u) {
      const int c = base + u * 128;
      if (c >= total) break;
      const int i = c / cpr, k0 = (c - i * cpr) * CE;
      if (SPLIT) {
        uint32_t hi[4], lo[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const __nv_bfloat162 h = __floats2bfloat162_rn(v[u][2 * q], v[u][2 * q + 1]);
          const float2 hf = __bfloat1622float2(h);
          const __nv_bfloat162 l = __floats2bfloat162_rn(v[u][2 * q] - hf.x, v[u][2 * q + 1] - hf.y);
          hi[q] = *reinterpret_cast<const uint32_t*>(&h);
          lo[q] = *reinterpret_cast<const uint32_t*>(&l);
        }
        const uint32_t o = swz(i, k0, 2);
        *reinterpret_cast<uint4*>(tile + o) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
        *reinterpret_cast<uint4*>(tile + Fmt<true>::plane_bytes + o) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
      } else {
        *reinterpret_cast<uint4*>(tile + swz(i, k0, 4)) =
            make_uint4(to_tf32(v[u][0]), to_tf32(v[u][1]), to_tf32(v[u][2]), to_tf32(v[u][3]));
      }
    }
  }
}

// Two warpgroups per CTA, each streaming its own images through the shared
// tensor pipe (while one restages or stores, the other's GEMM runs).  Warp w
// of warpgroup g owns TMEM lanes 32(w%4)..+31; slot g uses TMEM columns
// [256g, 256g+256): D1 and then D2 at +0, the restaged A operand at +128.
// The factor tile G is shared.
template <bool SPLIT>
__global__ void __launch_bounds__(256, 1)
    tc_conv2d_kernel(const float* __restrict__ in, float* __restrict__ out, long long nimg, int W,
                     int H, int Wp, int Hp, const float* __restrict__ G, int Gn, int* err) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* base = reinterpret_cast<uint8_t*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint8_t* g_tile = base;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int wg = warp >> 2, wt = tid & 127;
  uint8_t* x_tile = base + (1 + wg) * kTileBytes;
  uint64_t* bars = reinterpret_cast<uint64_t*>(base + 3 * kTileBytes);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(base + 3 * kTileBytes + 16);
  const uint32_t bar_a = ptx::smem_addr(&bars[wg]);
  const uint32_t g_a = ptx::smem_addr(g_tile), x_a = ptx::smem_addr(x_tile);

  load_factor<SPLIT>(g_tile, G, Gn, tid, blockDim.x);
  if (tid == 0) {
    ptx::mbar_init(ptx::smem_addr(&bars[0]), 1);
    ptx::mbar_init(ptx::smem_addr(&bars[1]), 1);
    ptx::fence_mbar_init();
  }
  if (warp == 0) ptx::tmem_alloc(ptx::smem_addr(tmem_slot), 2 * kTmemCols);
  ptx::fence_proxy_async_smem();
  ptx::tc_fence_before();
  __syncthreads();
  ptx::tc_fence_after();
  const uint32_t tmem = *tmem_slot + (uint32_t)wg * kTmemCols;
  // D1 and D2 share [0, 128); the second GEMM's A operand lives in [128, 256)
  const uint32_t d1 = tmem, d2 = tmem, a_hi = tmem + 128, a_lo = tmem + 192;
  const uint32_t lane_base = (uint32_t)((warp & 3) * 32) << 16;
  const int j = (warp & 3) * 32 + lane;  // x coordinate owned by this thread
  const bool vec = (W % 4) == 0 && (reinterpret_cast<uintptr_t>(in) & 15) == 0;
  uint32_t phase = 0;
  bool ok = true;

  for (long long img = 2 * (long long)blockIdx.x + wg; img < nimg && ok; img += 2LL * gridDim.x) {
    const float* src = in + (size_t)img * W * H;
    float* dst = out + (size_t)img * W * H;
    stage_image<SPLIT>(x_tile, src, W, H, Wp, Hp, wt, vec);
    ptx::fence_proxy_async_smem();
    wg_sync(wg);
    if (wt == 0) {
      ptx::tc_fence_after();
      issue_gemm<SPLIT>(d1, g_a, x_a, Wp, Hp);
      ptx::mma_commit(bar_a);
    }
    ok = wg_all(ptx::mbar_wait(bar_a, phase, kWaitNs), wg);
    phase ^= 1;
    ptx::tc_fence_after();
    // D1 -> the second GEMM's A operand (row j, K = i), kept in tensor memory
    for (int c0 = 0; c0 < Hp; c0 += 16) {
      float v[16];
      ptx::tmem_ld16(d1 + lane_base + (uint32_t)c0, v);
      ptx::tmem_ld_wait();
      restage16_tmem<SPLIT>(a_hi, a_lo, lane_base, c0, v);
    }
    ptx::tmem_st_wait();
    ptx::tc_fence_before();
    wg_sync(wg);
    if (wt == 0) {
      ptx::tc_fence_after();
      issue_gemm_ta<SPLIT>(d2, a_hi, a_lo, g_a, Hp, Hp);
      ptx::mma_commit(bar_a);
    }
    ok = wg_all(ok && ptx::mbar_wait(bar_a, phase, kWaitNs), wg);
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
    wg_sync(wg);
  }
  if (!ok && wt == 0) atomicExch(err, WDL_ERR_TIMEOUT);
  __syncthreads();
  ptx::tc_fence_after();
  if (warp == 0) ptx::tmem_dealloc(*tmem_slot, 2 * kTmemCols);
}

}  // namespace

// Tensor-core precisions: every grid with sides up to kTcMaxSide (2-D and 3-D,
// axis passes of conv_tc_axis.cu); 2-D grids with sides up to one 128-row tile
// also get the whole-image operator and the fused Sinkhorn kernel.
constexpr int kTcMaxSide = 512;

bool tc_supported(const wdl_ctx* ctx) {
  return ctx->W <= kTcMaxSide && ctx->H <= kTcMaxSide && ctx->D <= kTcMaxSide;
}

bool tc_fused(const wdl_ctx* ctx) { return ctx->tc != nullptr && ctx->tc->fused; }

int tc_init(wdl_ctx* ctx) {
  if (!tc_supported(ctx))
    return set_error(ctx, WDL_ERR_UNSUPPORTED, "tensor-core operator needs grid sides <= 512");
  auto* r = new TcResources();
  r->fused = ctx->ndim == 2 && ctx->W <= tc::kRows && ctx->H <= tc::kRows;
  r->smem_bytes = 3 * tc::kTileBytes + 1024 + 64;
  ctx->tc = r;
  WDL_CUDA_TRY(ctx, cudaMalloc(&r->d_err, sizeof(int)));
  WDL_CUDA_TRY(ctx, cudaMemset(r->d_err, 0, sizeof(int)));
  if (r->fused) {
    WDL_CUDA_TRY(ctx, cudaFuncSetAttribute(tc_conv2d_kernel<true>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)r->smem_bytes));
    WDL_CUDA_TRY(ctx, cudaFuncSetAttribute(tc_conv2d_kernel<false>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)r->smem_bytes));
  }
  return tc_axis_init(ctx, r->factor_blocks);
}

void tc_free(wdl_ctx* ctx) {
  if (!ctx->tc) return;
  if (ctx->tc->d_err) cudaFree(ctx->tc->d_err);
  for (auto* b : ctx->tc->factor_blocks)
    if (b) cudaFree(b);
  delete ctx->tc;
  ctx->tc = nullptr;
}

static int conv_stack_tc(wdl_ctx* ctx, const float* in, float* out, size_t nimg, cudaStream_t s) {
  const int W = ctx->W, H = ctx->H;
  const int Wp = (W + 15) & ~15, Hp = (H + 15) & ~15;
  const int Gn = W >= H ? W : H;
  const float* G = ctx->G32[W >= H ? 0 : 1];
  const size_t pairs = (nimg + 1) / 2;
  const unsigned grid = (unsigned)(pairs < (size_t)ctx->sm_count ? pairs : (size_t)ctx->sm_count);
  if (ctx->precision == WDL_SPLIT_BF16)
    tc_conv2d_kernel<true><<<grid, 256, ctx->tc->smem_bytes, s>>>(in, out, (long long)nimg, W, H, Wp,
                                                                  Hp, G, Gn, ctx->tc->d_err);
  else
    tc_conv2d_kernel<false><<<grid, 256, ctx->tc->smem_bytes, s>>>(in, out, (long long)nimg, W, H, Wp,
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
  int rc = ctx->tc->fused ? conv_stack_tc(ctx, in, out, nimg, s)
                          : conv_stack_tc_axes(ctx, in, out, tmp, nimg, ctx->tc->factor_blocks,
                                               ctx->tc->d_err, s);
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
  if (ctx->fused_sync) {
    int* sync = ctx->fused_sync;
    ctx->fused_sync = nullptr;
    int rc = sinkhorn_tc_status(ctx, sync);
    if (rc) return rc;
  }
  int h = 0;
  WDL_CUDA_TRY(ctx, cudaMemcpy(&h, ctx->tc->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (h != 0) {
    cudaMemset(ctx->tc->d_err, 0, sizeof(int));
    return set_error(ctx, h, "tensor-core kernel: a bounded wait timed out");
  }
  return WDL_OK;
}

}  // namespace wdl
