// Tensor-core (tcgen05) axis pass for grids whose sides exceed one 128-row
// tile, and for 3-D grids: the same primitive as the CUDA-core axis pass
// (conv_simt.cu), an image viewed as [R][C] (C contiguous) contracted along C
// with the dense C x C Gibbs factor and written as [C][R]:
//   out[c][r] = sum_k G[c][k] in[r][k]      (cpp/kernels.h:669-699, :762-807)
// Applying it once per axis returns the image to its layout, as the reference's
// x-pass into a transposed temporary followed by the y-pass (and z-pass).
//
// Each CTA computes a 128 (c) x TR (r) output tile of one image as a GEMM with
// M = 128 TMEM lanes = c, N = TR columns = r, K = C in chunks of 64: A = the
// factor rows c0.., B = the image rows r0.., both K-major in SMEM (128-byte
// swizzle), in one of two stages while the tensor cores work on the other.
// TR = 128 runs one CTA per SM (129 KB of SMEM); TR = 64 halves the image
// operand (97 KB) so two CTAs share an SM and hide each other's load latency,
// and splits the launch into twice as many, smaller tiles.  The tile height is
// chosen per shape by timing both on the call's own data.  The
// factor is prepared once per context as ready-made operand blocks (split into
// BF16 hi + lo, or rounded to TF32, already in the swizzled layout), so its
// blocks are plain 16-byte cp.async copies; the image rows are converted from
// FP32 by the CTA's threads.  The accumulator row of lane c holds
// out[c][r0..r0+TR-1], so each thread's epilogue stores are 64-byte contiguous
// runs of one output row.
//
// Precision as the 128-tile operator: kind::tf32, or split BF16 with
// hi*hi + hi*lo + lo*hi accumulated in FP32 (kind::f16).
#include <cuda.h>
#include <cudaTypedefs.h>

#include <cstring>

#include "tc_common.cuh"

namespace wdl {
namespace {

using namespace tc;

constexpr int kAxKc = 64;                  // K elements per chunk
constexpr int kAxTile = 128;               // output tile: 128 c x TR r
constexpr size_t kAxOperand = 32 * 1024;   // one 128 x 64 operand (both BF16 planes / TF32)
constexpr int kAxThreads = 256;

// Image operand of TR rows x 64 K elements: 128-byte column blocks of TR rows
// (TR * 128 bytes); two blocks (BF16 hi + lo planes, or TF32 K 0-31 / 32-63).
template <int TR>
struct AxGeom {
  static constexpr uint32_t kRegB = TR * 128;
  static constexpr size_t kBBytes = 2 * (size_t)kRegB;
  static constexpr size_t kStage = kAxOperand + kBBytes;  // A + B
  static constexpr size_t kSmem = 2 * kStage + 1024 + 64;
};

// Byte offset of element (r, k) in an operand whose 128-byte column blocks
// are REG bytes apart (the canonical 128-byte swizzle inside each block).
__device__ __forceinline__ uint32_t swz_reg(int r, int k, int esz, uint32_t reg) {
  const int per = 128 / esz;
  const int region = k / per;
  const int byte = (k - region * per) * esz;
  const int chunk = (byte >> 4) ^ (r & 7);
  return (uint32_t)(region * reg + r * 128 + (chunk << 4) + (byte & 15));
}

// 16-byte chunk (8 BF16 hi + 8 lo, or 4 TF32) of row r, elements k0.. of an
// operand whose BF16 lo plane starts REG bytes after the hi plane.
template <bool SPLIT, uint32_t REG>
__device__ __forceinline__ void put_axis_chunk(uint8_t* tile, int r, int k0, const float* v) {
  if (SPLIT) {
    uint32_t hi[4], lo[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const __nv_bfloat162 h = __floats2bfloat162_rn(v[2 * q], v[2 * q + 1]);
      const float2 hf = __bfloat1622float2(h);
      const __nv_bfloat162 l = __floats2bfloat162_rn(v[2 * q] - hf.x, v[2 * q + 1] - hf.y);
      hi[q] = *reinterpret_cast<const uint32_t*>(&h);
      lo[q] = *reinterpret_cast<const uint32_t*>(&l);
    }
    const uint32_t o = swz_reg(r, k0, 2, REG);
    *reinterpret_cast<uint4*>(tile + o) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
    *reinterpret_cast<uint4*>(tile + REG + o) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
  } else {
    *reinterpret_cast<uint4*>(tile + swz_reg(r, k0, 4, REG)) =
        make_uint4(to_tf32(v[0]), to_tf32(v[1]), to_tf32(v[2]), to_tf32(v[3]));
  }
}

// Rows 0.. (at most `rows` valid) of a row-major matrix with `len` elements
// per row, elements kb..kb+63 (zero beyond len): loaded into registers by
// load_operand, converted and stored into a 128 x 64 operand by
// store_operand, so the loads of the next chunk can be in flight while the
// current one is converted and multiplied.
template <bool SPLIT, int TR>
struct OperandRegs {
  static constexpr int CE = SPLIT ? 8 : 4;
  static constexpr int CPR = kAxKc / CE;            // chunks per row
  static constexpr int PER = TR * CPR / kAxThreads;  // chunks per thread
  float v[PER][CE];
};

template <bool SPLIT, int TR>
__device__ __forceinline__ void load_operand(OperandRegs<SPLIT, TR>& o, const float* __restrict__ src, int rows,
                                             int len, int kb, bool vec, int t) {
  using O = OperandRegs<SPLIT, TR>;
#pragma unroll
  for (int u = 0; u < O::PER; ++u) {
    const int c = t + u * kAxThreads;
    const int r = c / O::CPR, k0 = kb + (c - r * O::CPR) * O::CE;
    const float* row = src + (size_t)r * len;
    if (r < rows && vec && k0 + O::CE <= len) {
#pragma unroll
      for (int q = 0; q < O::CE; q += 4) {
        const float4 f = __ldg(reinterpret_cast<const float4*>(row + k0 + q));
        o.v[u][q] = f.x; o.v[u][q + 1] = f.y; o.v[u][q + 2] = f.z; o.v[u][q + 3] = f.w;
      }
    } else {
#pragma unroll
      for (int q = 0; q < O::CE; ++q) o.v[u][q] = (r < rows && k0 + q < len) ? __ldg(row + k0 + q) : 0.f;
    }
  }
}

template <bool SPLIT, int TR>
__device__ __forceinline__ void store_operand(uint8_t* tile, const OperandRegs<SPLIT, TR>& o, int t) {
  using O = OperandRegs<SPLIT, TR>;
#pragma unroll
  for (int u = 0; u < O::PER; ++u) {
    const int c = t + u * kAxThreads;
    const int r = c / O::CPR, kk = (c - r * O::CPR) * O::CE;
    put_axis_chunk<SPLIT, AxGeom<TR>::kRegB>(tile, r, kk, o.v[u]);
  }
}

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// The factor of one axis (C x C) as operand blocks: block (m, j) holds rows
// 128m.. and K elements 64j.. in the SMEM layout of a 128 x 64 operand.
template <bool SPLIT>
__global__ void k_build_factor_blocks(const float* __restrict__ G, int C, uint8_t* __restrict__ blocks) {
  const int nch = (C + kAxKc - 1) / kAxKc;
  const int m = blockIdx.x / nch, j = blockIdx.x - m * nch;
  uint8_t* tile = blocks + (size_t)blockIdx.x * kAxOperand;
  const int c0 = m * kAxTile;
  constexpr int CE = SPLIT ? 8 : 4;
  constexpr int CPR = kAxKc / CE;
  for (int c = threadIdx.x; c < kAxTile * CPR; c += blockDim.x) {
    const int r = c / CPR, kk = (c - r * CPR) * CE;
    float v[CE];
    for (int q = 0; q < CE; ++q) {
      const int row = c0 + r, k = j * kAxKc + kk + q;
      v[q] = (row < C && k < C) ? G[(size_t)row * C + k] : 0.f;
    }
    put_axis_chunk<SPLIT, kRegionBytes>(tile, r, kk, v);
  }
}

template <bool SPLIT, int TR>
__global__ void __launch_bounds__(kAxThreads, TR == 64 ? 2 : 1)
    tc_axis_kernel(const float* __restrict__ in, float* __restrict__ out,
                   const uint8_t* __restrict__ gblocks, int R, int C, size_t img_stride, int reach, int* err) {
  using Ge = AxGeom<TR>;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* bars = reinterpret_cast<uint64_t*>(base + 2 * Ge::kStage);  // [2]
  uint32_t* tslot = reinterpret_cast<uint32_t*>(base + 2 * Ge::kStage + 16);
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const int c0 = blockIdx.x * kAxTile, r0 = blockIdx.y * TR;
  const float* src = in + (size_t)blockIdx.z * img_stride + (size_t)r0 * C;
  const int nch = (C + kAxKc - 1) / kAxKc;
  const uint8_t* gsrc = gblocks + (size_t)blockIdx.x * nch * kAxOperand;
  // K chunks whose factor rows c0.. are not all zero: |c - k| <= reach.  The
  // other chunks' FP32 factor entries (hence their BF16 / TF32 operands) are
  // exactly zero and add exactly nothing, so they are neither loaded nor
  // multiplied.
  const int c_last = min(c0 + kAxTile, C) - 1;
  const int jlo = max(0, c0 - reach) / kAxKc;
  const int jhi = min(C - 1, c_last + reach) / kAxKc + 1;
  float* dst = out + (size_t)blockIdx.z * img_stride;
  const int b_rows = min(TR, R - r0);
  const bool vec = (C & 3) == 0;

  if (t == 0) {
    ptx::mbar_init(ptx::smem_addr(&bars[0]), 1);
    ptx::mbar_init(ptx::smem_addr(&bars[1]), 1);
    ptx::fence_mbar_init();
  }
  if (warp == 0) ptx::tmem_alloc(ptx::smem_addr(tslot), TR);
  ptx::tc_fence_before();
  __syncthreads();
  ptx::tc_fence_after();
  const uint32_t d = *tslot;

  using F = Fmt<SPLIT>;
  const uint32_t id = ptx::idesc(F::fmt, 128, TR);
  bool ok = true;
  OperandRegs<SPLIT, TR> breg;
  load_operand<SPLIT, TR>(breg, src, b_rows, C, jlo * kAxKc, vec, t);
  for (int j = jlo; j < jhi; ++j) {
    const int jj = j - jlo;  // position in this CTA's chunk sequence
    const int st = jj & 1;
    uint8_t* a_tile = base + st * Ge::kStage;
    uint8_t* b_tile = a_tile + kAxOperand;
    if (jj >= 2) {  // the MMAs of chunk jj-2 read this stage: wait for their commit
      const bool w = t != 0 || ptx::mbar_wait(ptx::smem_addr(&bars[st]), (uint32_t)(((jj - 2) >> 1) & 1), kWaitNs);
      ok = __syncthreads_and(w) != 0;
      if (!ok) break;
    }
    {  // factor block: 32 KB, 8 x 16 bytes per thread, straight copies
      const uint8_t* gb = gsrc + (size_t)j * kAxOperand;
      const uint32_t a_s = ptx::smem_addr(a_tile);
#pragma unroll
      for (int u = 0; u < (int)(kAxOperand / 16 / kAxThreads); ++u) {
        const int o = (t + u * kAxThreads) * 16;
        cp_async16(a_s + o, gb + o);
      }
      cp_async_commit();
    }
    store_operand<SPLIT, TR>(b_tile, breg, t);
    if (j + 1 < jhi) load_operand<SPLIT, TR>(breg, src, b_rows, C, (j + 1) * kAxKc, vec, t);
    cp_async_wait_all();
    ptx::fence_proxy_async_smem();
    ptx::tc_fence_before();
    __syncthreads();
    if (t == 0) {
      ptx::tc_fence_after();
      const uint32_t a = ptx::smem_addr(a_tile), b = ptx::smem_addr(b_tile);
      const int steps = kAxKc / F::kstep;
#pragma unroll
      for (int ks = 0; ks < steps; ++ks) {
        const uint32_t byte = (uint32_t)ks * 32u;
        const uint32_t offa = (byte >> 7) * kRegionBytes + (byte & 127u);
        const uint32_t offb = (byte >> 7) * Ge::kRegB + (byte & 127u);
        const uint32_t acc = (jj > 0 || ks > 0) ? 1u : 0u;
        const uint64_t ad = ptx::sw128_desc(a + offa), bd = ptx::sw128_desc(b + offb);
        if (SPLIT) {
          const uint64_t alo = ptx::sw128_desc(a + kRegionBytes + offa);
          const uint64_t blo = ptx::sw128_desc(b + Ge::kRegB + offb);
          ptx::mma_bf16(d, ad, bd, id, acc);
          ptx::mma_bf16(d, ad, blo, id, 1u);
          ptx::mma_bf16(d, alo, bd, id, 1u);
        } else {
          ptx::mma_tf32(d, ad, bd, id, acc);
        }
      }
      ptx::mma_commit(ptx::smem_addr(&bars[st]));
    }
  }
  if (ok) {  // the last commit covers every MMA issued before it
    const int jj = jhi - 1 - jlo;
    const bool w = t != 0 || ptx::mbar_wait(ptx::smem_addr(&bars[jj & 1]), (uint32_t)((jj >> 1) & 1), kWaitNs);
    ok = __syncthreads_and(w) != 0;
  }
  if (!ok) {
    if (t == 0) atomicExch(err, WDL_ERR_TIMEOUT);
  } else {
    ptx::tc_fence_after();
    const int q = warp & 3, half = warp >> 2;
    const int c = c0 + q * 32 + lane;
    const bool rvec = (R & 3) == 0;
#pragma unroll
    for (int cc = 0; cc < TR / 32; ++cc) {
      float v[16];
      const int col = half * (TR / 2) + cc * 16;
      ptx::tmem_ld16(d + ((uint32_t)(q * 32) << 16) + (uint32_t)col, v);
      ptx::tmem_ld_wait();
      if (c < C) {
        float* orow = dst + (size_t)c * R;
        const int rb = r0 + col;
#pragma unroll
        for (int i = 0; i < 16; i += 4) {
          const int r = rb + i;
          if (rvec && r + 3 < R) {
            *reinterpret_cast<float4*>(orow + r) = make_float4(v[i], v[i + 1], v[i + 2], v[i + 3]);
          } else {
            for (int e = 0; e < 4; ++e)
              if (r + e < R) orow[r + e] = v[i + e];
          }
        }
      }
    }
  }
  ptx::tc_fence_before();
  __syncthreads();
  ptx::tc_fence_after();
  if (warp == 0) ptx::tmem_dealloc(d, TR);
}

// ---- copy-engine staged form ---------------------------------------------------------
// The same output tile, K chunks (band-limited as above) and MMAs as
// tc_axis_kernel, with both operands staged by the copy engine instead of the
// CTA's loads: per K chunk, one tiled TMA load brings the FP32 image rows
// r0..r0+TR-1, elements kb..kb+63 (zero outside the tensor), and one bulk copy
// the ready-made factor block, into a ring of S stages that complete on one
// transaction-count barrier each.  One thread keeps S-1 chunks in flight ahead
// of the one being multiplied; the CTA's threads only convert the landed FP32
// rows (SMEM -> BF16 hi/lo or TF32 operand, double-buffered) while the tensor
// cores multiply the previous chunk.  The image is viewed as the 2-D tensor
// [images * R][C] (row pitch C * 4 bytes, so C % 4 == 0 and a 16-byte aligned
// base are required; other shapes take tc_axis_kernel).  The converted values,
// the chunk order and the MMA sequence are tc_axis_kernel's, so both forms give
// the same bits.  No multicast: every load reads this GPU's own memory for one
// CTA.
template <int TR>
struct AxTmaGeom {
  static constexpr int kStages = TR == 64 ? 3 : 2;
  static constexpr uint32_t kRaw = TR * kAxKc * 4;  // FP32 rows of one chunk
  static constexpr uint32_t kRegB = TR * 128;       // one 128-byte column block of the operand
  static constexpr uint32_t kB = 2 * kRegB;         // converted operand (both planes / TF32 K 0-63)
  static constexpr size_t kRaw0 = (size_t)kStages * kAxOperand;
  static constexpr size_t kB0 = kRaw0 + (size_t)kStages * kRaw;
  static constexpr size_t kBar0 = kB0 + 2 * (size_t)kB;
  static constexpr size_t kSmem = kBar0 + 128 + 1024;
};

template <bool SPLIT, int TR>
__global__ void __launch_bounds__(kAxThreads, 1)
    tc_axis_tma_kernel(const __grid_constant__ CUtensorMap tmap, float* __restrict__ out,
                       const uint8_t* __restrict__ gblocks, int R, int C, size_t img_stride, int reach, int* err) {
  using Ge = AxTmaGeom<TR>;
  constexpr int S = Ge::kStages;
  using F = Fmt<SPLIT>;
  constexpr int CE = SPLIT ? 8 : 4;
  constexpr int CPR = kAxKc / CE;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(base + Ge::kBar0);  // [S] copies of a stage landed
  uint64_t* mmab = full + S;                                       // [2] MMAs reading operand b done
  uint32_t* tslot = reinterpret_cast<uint32_t*>(mmab + 2);
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const int c0 = blockIdx.x * kAxTile, r0 = blockIdx.y * TR;
  const int nch = (C + kAxKc - 1) / kAxKc;
  const uint8_t* gsrc = gblocks + (size_t)blockIdx.x * nch * kAxOperand;
  float* dst = out + (size_t)blockIdx.z * img_stride;
  const int c_last = min(c0 + kAxTile, C) - 1;
  const int jlo = max(0, c0 - reach) / kAxKc;
  const int n = min(C - 1, c_last + reach) / kAxKc + 1 - jlo;
  const int ybase = (int)blockIdx.z * R + r0;  // row of the 2-D view

  if (t == 0) {
    for (int q = 0; q < S; ++q) ptx::mbar_init(ptx::smem_addr(&full[q]), 1);
    ptx::mbar_init(ptx::smem_addr(&mmab[0]), 1);
    ptx::mbar_init(ptx::smem_addr(&mmab[1]), 1);
    ptx::fence_mbar_init();
  }
  if (warp == 0) ptx::tmem_alloc(ptx::smem_addr(tslot), TR);
  ptx::tc_fence_before();
  __syncthreads();
  ptx::tc_fence_after();
  const uint32_t d = *tslot;
  const uint32_t id = ptx::idesc(F::fmt, 128, TR);

  auto a_tile = [&](int q) { return base + (size_t)q * kAxOperand; };
  auto raw_tile = [&](int q) { return base + Ge::kRaw0 + (size_t)q * Ge::kRaw; };
  auto b_tile = [&](int b) { return base + Ge::kB0 + (size_t)b * Ge::kB; };
  // thread 0: the copies of chunk jj into stage jj % S
  auto issue = [&](int jj) {
    const int q = jj % S;
    const uint32_t bar = ptx::smem_addr(&full[q]);
    ptx::mbar_arrive_expect_tx(bar, (uint32_t)kAxOperand + Ge::kRaw);
    ptx::bulk_load(ptx::smem_addr(a_tile(q)), gsrc + (size_t)(jlo + jj) * kAxOperand, (uint32_t)kAxOperand, bar);
    ptx::tma_load_2d(ptx::smem_addr(raw_tile(q)), &tmap, (jlo + jj) * kAxKc, ybase, bar);
  };
  int issued = 0;
  if (t == 0)
    for (; issued < S && issued < n; ++issued) issue(issued);

  bool ok = true;
  int jj = 0;
  for (; jj < n; ++jj) {
    const int q = jj % S, b = jj & 1;
    // this chunk's copies have landed; the operand buffer b is no longer read
    // by the MMAs of chunk jj - 2
    bool w = ptx::mbar_wait(ptx::smem_addr(&full[q]), (uint32_t)((jj / S) & 1), kWaitNs);
    if (jj >= 2) w = w && ptx::mbar_wait(ptx::smem_addr(&mmab[b]), (uint32_t)(((jj - 2) >> 1) & 1), kWaitNs);
    ok = __syncthreads_and(w) != 0;
    if (!ok) break;
    {  // landed FP32 rows -> the operand (rows beyond the image are never stored)
      const float* raw = reinterpret_cast<const float*>(raw_tile(q));
      uint8_t* bt = b_tile(b);
#pragma unroll
      for (int u = 0; u < TR * CPR / kAxThreads; ++u) {
        const int c = t + u * kAxThreads;
        const int r = c / CPR, kk = (c - r * CPR) * CE;
        float v[CE];
#pragma unroll
        for (int e = 0; e < CE; e += 4) {
          const float4 f = *reinterpret_cast<const float4*>(raw + r * kAxKc + kk + e);
          v[e] = f.x; v[e + 1] = f.y; v[e + 2] = f.z; v[e + 3] = f.w;
        }
        put_axis_chunk<SPLIT, Ge::kRegB>(bt, r, kk, v);
      }
    }
    ptx::fence_proxy_async_smem();
    ptx::tc_fence_before();
    __syncthreads();
    if (t == 0) {
      ptx::tc_fence_after();
      const uint32_t a = ptx::smem_addr(a_tile(q)), bb = ptx::smem_addr(b_tile(b));
      const int steps = kAxKc / F::kstep;
#pragma unroll
      for (int ks = 0; ks < steps; ++ks) {
        const uint32_t byte = (uint32_t)ks * 32u;
        const uint32_t offa = (byte >> 7) * kRegionBytes + (byte & 127u);
        const uint32_t offb = (byte >> 7) * Ge::kRegB + (byte & 127u);
        const uint32_t acc = (jj > 0 || ks > 0) ? 1u : 0u;
        const uint64_t ad = ptx::sw128_desc(a + offa), bd = ptx::sw128_desc(bb + offb);
        if (SPLIT) {
          const uint64_t alo = ptx::sw128_desc(a + kRegionBytes + offa);
          const uint64_t blo = ptx::sw128_desc(bb + Ge::kRegB + offb);
          ptx::mma_bf16(d, ad, bd, id, acc);
          ptx::mma_bf16(d, ad, blo, id, 1u);
          ptx::mma_bf16(d, alo, bd, id, 1u);
        } else {
          ptx::mma_tf32(d, ad, bd, id, acc);
        }
      }
      ptx::mma_commit(ptx::smem_addr(&mmab[b]));
      // refill the stage of chunk jj - 1 once its MMAs are done (its factor
      // block is read by them; its FP32 rows were converted last iteration)
      if (jj >= 1 && issued < n) {
        if (ptx::mbar_wait(ptx::smem_addr(&mmab[(jj - 1) & 1]), (uint32_t)(((jj - 1) >> 1) & 1), kWaitNs)) {
          issue(issued);
          ++issued;
        } else {
          atomicExch(err, WDL_ERR_TIMEOUT);
        }
      }
    }
  }
  if (ok) {  // the last commit covers every MMA issued before it
    const int last = n - 1;
    const bool w = t != 0 || ptx::mbar_wait(ptx::smem_addr(&mmab[last & 1]), (uint32_t)((last >> 1) & 1), kWaitNs);
    ok = __syncthreads_and(w) != 0;
  }
  if (!ok) {
    if (t == 0) {
      atomicExch(err, WDL_ERR_TIMEOUT);
      // let the copies still in flight land (bounded) before the CTA's SMEM goes away
      for (int p = jj; p < issued; ++p)
        ptx::mbar_wait(ptx::smem_addr(&full[p % S]), (uint32_t)((p / S) & 1), kWaitNs);
      if (jj >= 1)
        ptx::mbar_wait(ptx::smem_addr(&mmab[(jj - 1) & 1]), (uint32_t)(((jj - 1) >> 1) & 1), kWaitNs);
    }
    __syncthreads();
  } else {
    ptx::tc_fence_after();
    const int qd = warp & 3, half = warp >> 2;
    const int c = c0 + qd * 32 + lane;
    const bool rvec = (R & 3) == 0;
#pragma unroll
    for (int cc = 0; cc < TR / 32; ++cc) {
      float v[16];
      const int col = half * (TR / 2) + cc * 16;
      ptx::tmem_ld16(d + ((uint32_t)(qd * 32) << 16) + (uint32_t)col, v);
      ptx::tmem_ld_wait();
      if (c < C) {
        float* orow = dst + (size_t)c * R;
        const int rb = r0 + col;
#pragma unroll
        for (int i = 0; i < 16; i += 4) {
          const int r = rb + i;
          if (rvec && r + 3 < R) {
            *reinterpret_cast<float4*>(orow + r) = make_float4(v[i], v[i + 1], v[i + 2], v[i + 3]);
          } else {
            for (int e = 0; e < 4; ++e)
              if (r + e < R) orow[r + e] = v[i + e];
          }
        }
      }
    }
  }
  ptx::tc_fence_before();
  __syncthreads();
  ptx::tc_fence_after();
  if (warp == 0) ptx::tmem_dealloc(d, TR);
}

// ---- persistent, factor-resident form ------------------------------------------------
// A CTA owns one 128-row slab c0.. of the factor and keeps its band-limited K
// chunks resident in SMEM (loaded once by bulk copies), then walks a strided
// share of the (image, 64-row tile) pairs: per tile and chunk one TMA load of
// the FP32 image rows (two stages), the conversion into the operand (two
// buffers) and the MMAs into one of two TMEM accumulators, so that a tile's
// epilogue (TMEM -> its output rows) runs while the tensor cores work on the
// next tile.  The per-tile factor reloads of the tiled forms (4 of every 6 bytes
// they move) disappear.  Same operand values, chunk order and MMAs per output
// tile as the other forms, so the same bits.
constexpr int kPxTR = 64;         // image rows per tile (MMA N)
constexpr int kPxMaxChunks = 5;   // resident factor chunks (5 x 32 KB)
struct PxGeom {
  static constexpr uint32_t kRaw = kPxTR * kAxKc * 4;   // 16 KB
  static constexpr uint32_t kRegB = kPxTR * 128;
  static constexpr uint32_t kB = 2 * kRegB;             // 16 KB
  static constexpr size_t kRaw0 = (size_t)kPxMaxChunks * kAxOperand;
  static constexpr size_t kB0 = kRaw0 + 2 * (size_t)kRaw;
  static constexpr size_t kBar0 = kB0 + 2 * (size_t)kB;
  static constexpr size_t kSmem = kBar0 + 128 + 1024;
};

template <bool SPLIT>
__global__ void __launch_bounds__(kAxThreads, 1)
    tc_axis_persist_kernel(const __grid_constant__ CUtensorMap tmap, float* __restrict__ out,
                           const uint8_t* __restrict__ gblocks, int R, int C, int nimg, size_t img_stride,
                           int reach, int* err) {
  using Ge = PxGeom;
  using F = Fmt<SPLIT>;
  constexpr int CE = SPLIT ? 8 : 4;
  constexpr int CPR = kAxKc / CE;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(base + Ge::kBar0);  // [2] image chunk landed
  uint64_t* mmab = full + 2;                                       // [2] MMAs reading operand b done
  uint64_t* fbar = mmab + 2;                                       // factor slab landed
  uint32_t* tslot = reinterpret_cast<uint32_t*>(fbar + 1);
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const int c0 = blockIdx.x * kAxTile;
  const int nch = (C + kAxKc - 1) / kAxKc;
  const int c_last = min(c0 + kAxTile, C) - 1;
  const int jlo = max(0, c0 - reach) / kAxKc;
  const int nk = min(C - 1, c_last + reach) / kAxKc + 1 - jlo;  // <= kPxMaxChunks (host-checked)
  const int rtiles = (R + kPxTR - 1) / kPxTR;
  const int ntile_all = nimg * rtiles;
  // this CTA's tiles: blockIdx.y, blockIdx.y + gridDim.y, ...
  const int my_tiles = blockIdx.y < ntile_all ? (ntile_all - 1 - (int)blockIdx.y) / (int)gridDim.y + 1 : 0;
  const int nsteps = my_tiles * nk;

  if (t == 0) {
    ptx::mbar_init(ptx::smem_addr(&full[0]), 1);
    ptx::mbar_init(ptx::smem_addr(&full[1]), 1);
    ptx::mbar_init(ptx::smem_addr(&mmab[0]), 1);
    ptx::mbar_init(ptx::smem_addr(&mmab[1]), 1);
    ptx::mbar_init(ptx::smem_addr(fbar), 1);
    ptx::fence_mbar_init();
  }
  if (warp == 0) ptx::tmem_alloc(ptx::smem_addr(tslot), 2 * kPxTR);
  ptx::tc_fence_before();
  __syncthreads();
  ptx::tc_fence_after();
  const uint32_t d0 = *tslot;
  const uint32_t id = ptx::idesc(F::fmt, 128, kPxTR);

  auto raw_tile = [&](int q) { return base + Ge::kRaw0 + (size_t)q * Ge::kRaw; };
  auto b_tile = [&](int b) { return base + Ge::kB0 + (size_t)b * Ge::kB; };
  // step g = (tile i, chunk jj): its image chunk into raw stage g & 1
  auto issue = [&](int g) {
    const int i = g / nk, jj = g - i * nk;
    const int tile = (int)blockIdx.y + i * (int)gridDim.y;
    const int z = tile / rtiles, r0 = (tile - z * rtiles) * kPxTR;
    const uint32_t bar = ptx::smem_addr(&full[g & 1]);
    ptx::mbar_arrive_expect_tx(bar, Ge::kRaw);
    ptx::tma_load_2d(ptx::smem_addr(raw_tile(g & 1)), &tmap, (jlo + jj) * kAxKc, z * R + r0, bar);
  };
  int issued = 0, committed = 0;  // thread 0: image chunks requested, steps whose MMAs are issued
  if (t == 0 && nsteps > 0) {
    const uint32_t fb = ptx::smem_addr(fbar);
    ptx::mbar_arrive_expect_tx(fb, (uint32_t)(nk * kAxOperand));
    const uint8_t* gsrc = gblocks + ((size_t)blockIdx.x * nch + jlo) * kAxOperand;
    for (int jj = 0; jj < nk; ++jj)
      ptx::bulk_load(ptx::smem_addr(base + (size_t)jj * kAxOperand), gsrc + (size_t)jj * kAxOperand,
                     (uint32_t)kAxOperand, fb);
    for (; issued < 2 && issued < nsteps; ++issued) issue(issued);
  }
  bool ok = nsteps == 0 || __syncthreads_and(t != 0 || ptx::mbar_wait(ptx::smem_addr(fbar), 0, kWaitNs)) != 0;

  // epilogue of tile i (accumulator i & 1): TMEM -> out[c][r0 ..]
  auto epilogue = [&](int i) {
    const int tile = (int)blockIdx.y + i * (int)gridDim.y;
    const int z = tile / rtiles, r0 = (tile - z * rtiles) * kPxTR;
    float* dst = out + (size_t)z * img_stride;
    const uint32_t d = d0 + (uint32_t)((i & 1) * kPxTR);
    const int qd = warp & 3, half = warp >> 2;
    const int c = c0 + qd * 32 + lane;
    const bool rvec = (R & 3) == 0;
#pragma unroll
    for (int cc = 0; cc < kPxTR / 32; ++cc) {
      float v[16];
      const int col = half * (kPxTR / 2) + cc * 16;
      ptx::tmem_ld16(d + ((uint32_t)(qd * 32) << 16) + (uint32_t)col, v);
      ptx::tmem_ld_wait();
      if (c < C) {
        float* orow = dst + (size_t)c * R;
        const int rb = r0 + col;
#pragma unroll
        for (int e = 0; e < 16; e += 4) {
          const int r = rb + e;
          if (rvec && r + 3 < R) {
            *reinterpret_cast<float4*>(orow + r) = make_float4(v[e], v[e + 1], v[e + 2], v[e + 3]);
          } else {
            for (int q = 0; q < 4; ++q)
              if (r + q < R) orow[r + q] = v[e + q];
          }
        }
      }
    }
  };

  int g = 0;
  for (; ok && g < nsteps; ++g) {
    const int i = g / nk, jj = g - i * nk, b = g & 1;
    bool w = ptx::mbar_wait(ptx::smem_addr(&full[g & 1]), (uint32_t)((g >> 1) & 1), kWaitNs);
    if (g >= 2) w = w && ptx::mbar_wait(ptx::smem_addr(&mmab[b]), (uint32_t)(((g - 2) >> 1) & 1), kWaitNs);
    ok = __syncthreads_and(w) != 0;
    if (!ok) break;
    {  // landed FP32 rows -> the operand
      const float* raw = reinterpret_cast<const float*>(raw_tile(g & 1));
      uint8_t* bt = b_tile(b);
#pragma unroll
      for (int u = 0; u < kPxTR * CPR / kAxThreads; ++u) {
        const int cidx = t + u * kAxThreads;
        const int r = cidx / CPR, kk = (cidx - r * CPR) * CE;
        float v[CE];
#pragma unroll
        for (int e = 0; e < CE; e += 4) {
          const float4 f4 = *reinterpret_cast<const float4*>(raw + r * kAxKc + kk + e);
          v[e] = f4.x; v[e + 1] = f4.y; v[e + 2] = f4.z; v[e + 3] = f4.w;
        }
        put_axis_chunk<SPLIT, Ge::kRegB>(bt, r, kk, v);
      }
    }
    ptx::fence_proxy_async_smem();
    ptx::tc_fence_before();
    __syncthreads();
    if (t == 0) {
      ptx::tc_fence_after();
      // the raw stage is converted: refill it with step g + 2
      if (issued < nsteps) {
        issue(issued);
        ++issued;
      }
      const uint32_t a = ptx::smem_addr(base + (size_t)jj * kAxOperand), bb = ptx::smem_addr(b_tile(b));
      const uint32_t d = d0 + (uint32_t)((i & 1) * kPxTR);
      const int steps = kAxKc / F::kstep;
#pragma unroll
      for (int ks = 0; ks < steps; ++ks) {
        const uint32_t byte = (uint32_t)ks * 32u;
        const uint32_t offa = (byte >> 7) * kRegionBytes + (byte & 127u);
        const uint32_t offb = (byte >> 7) * Ge::kRegB + (byte & 127u);
        const uint32_t acc = (jj > 0 || ks > 0) ? 1u : 0u;
        const uint64_t ad = ptx::sw128_desc(a + offa), bd = ptx::sw128_desc(bb + offb);
        if (SPLIT) {
          const uint64_t alo = ptx::sw128_desc(a + kRegionBytes + offa);
          const uint64_t blo = ptx::sw128_desc(bb + Ge::kRegB + offb);
          ptx::mma_bf16(d, ad, bd, id, acc);
          ptx::mma_bf16(d, ad, blo, id, 1u);
          ptx::mma_bf16(d, alo, bd, id, 1u);
        } else {
          ptx::mma_tf32(d, ad, bd, id, acc);
        }
      }
      ptx::mma_commit(ptx::smem_addr(&mmab[b]));
      ++committed;
    }
    // the previous tile's accumulator is complete once the MMAs of its last
    // chunk (step g - 1) are: store it while this tile's chunks multiply
    if (jj == 0 && i > 0) {
      const bool we = t != 0 || ptx::mbar_wait(ptx::smem_addr(&mmab[(g - 1) & 1]), (uint32_t)(((g - 1) >> 1) & 1), kWaitNs);
      ok = __syncthreads_and(we) != 0;
      if (!ok) break;
      ptx::tc_fence_after();
      epilogue(i - 1);
      // the next MMAs into this accumulator (tile i + 1) come after this sync
      ptx::tc_fence_before();
      __syncthreads();
    }
  }
  if (ok && nsteps > 0) {  // the last tile
    const int last = nsteps - 1;
    const bool w = t != 0 || ptx::mbar_wait(ptx::smem_addr(&mmab[last & 1]), (uint32_t)((last >> 1) & 1), kWaitNs);
    ok = __syncthreads_and(w) != 0;
    if (ok) {
      ptx::tc_fence_after();
      epilogue(my_tiles - 1);
    }
  }
  if (!ok) {
    if (t == 0) {
      atomicExch(err, WDL_ERR_TIMEOUT);
      // let copies and MMAs still in flight finish (bounded) before the SMEM and TMEM go away
      ptx::mbar_wait(ptx::smem_addr(fbar), 0, kWaitNs);
      for (int q = g; q < issued; ++q) ptx::mbar_wait(ptx::smem_addr(&full[q & 1]), (uint32_t)((q >> 1) & 1), kWaitNs);
      if (committed >= 1)
        ptx::mbar_wait(ptx::smem_addr(&mmab[(committed - 1) & 1]), (uint32_t)(((committed - 1) >> 1) & 1), kWaitNs);
    }
    __syncthreads();
  }
  ptx::tc_fence_before();
  __syncthreads();
  ptx::tc_fence_after();
  if (warp == 0) ptx::tmem_dealloc(d0, 2 * kPxTR);
}

// cuTensorMapEncodeTiled from the driver, looked up once through the runtime.
PFN_cuTensorMapEncodeTiled_v12000 encode_tiled() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      p = nullptr;
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }();
  return fn;
}

// The copy-engine form applies: row pitch and base 16-byte aligned.
bool tc_axis_tma_ok(const float* in, int C) {
  return (C % 4) == 0 && (reinterpret_cast<uintptr_t>(in) % 16) == 0 && encode_tiled() != nullptr;
}

template <int TR>
int tc_axis_tma_launch(wdl_ctx* ctx, const float* in, float* out, const uint8_t* G, int R, int C, size_t nimg,
                       size_t img_stride, int reach, int* err, cudaStream_t s) {
  size_t done = 0;
  while (done < nimg) {
    size_t chunk = nimg - done;
    if (chunk > 65535) chunk = 65535;
    const float* src = in + done * img_stride;
    // the chunk's images as the 2-D tensor [chunk * R][C] (image stride R * C)
    CUtensorMap tmap;
    const cuuint64_t dims[2] = {(cuuint64_t)C, (cuuint64_t)chunk * (cuuint64_t)R};
    const cuuint64_t strides[1] = {(cuuint64_t)C * sizeof(float)};
    const cuuint32_t box[2] = {(cuuint32_t)kAxKc, (cuuint32_t)TR};
    const cuuint32_t estr[2] = {1, 1};
    if (img_stride != (size_t)R * C)
      return set_error(ctx, WDL_ERR_UNSUPPORTED, "copy-engine axis pass: images must be contiguous");
    const CUresult cr = encode_tiled()(&tmap, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(src), dims,
                                       strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                       CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                                       CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (cr != CUDA_SUCCESS) return set_error(ctx, WDL_ERR_CUDA, "cuTensorMapEncodeTiled failed");
    dim3 grid((C + kAxTile - 1) / kAxTile, (R + TR - 1) / TR, (unsigned)chunk);
    const size_t smem = AxTmaGeom<TR>::kSmem;
    if (ctx->precision == WDL_SPLIT_BF16)
      tc_axis_tma_kernel<true, TR><<<grid, kAxThreads, smem, s>>>(tmap, out + done * img_stride, G, R, C,
                                                                  img_stride, reach, err);
    else
      tc_axis_tma_kernel<false, TR><<<grid, kAxThreads, smem, s>>>(tmap, out + done * img_stride, G, R, C,
                                                                   img_stride, reach, err);
    WDL_LAUNCH_CHECK(ctx);
    done += chunk;
  }
  return WDL_OK;
}

// The factor-resident form applies when every slab's band-limited chunks fit
// the resident buffer (and the copy-engine form applies).
bool tc_axis_persist_ok(const float* in, int C, int reach) {
  if (!tc_axis_tma_ok(in, C)) return false;
  for (int c0 = 0; c0 < C; c0 += kAxTile) {
    const int c_last = (c0 + kAxTile < C ? c0 + kAxTile : C) - 1;
    const int lo = (c0 - reach > 0 ? c0 - reach : 0) / kAxKc;
    const int hi = (c_last + reach < C - 1 ? c_last + reach : C - 1) / kAxKc + 1;
    if (hi - lo > kPxMaxChunks) return false;
  }
  return true;
}

int tc_axis_persist_launch(wdl_ctx* ctx, const float* in, float* out, const uint8_t* G, int R, int C,
                           size_t nimg, size_t img_stride, int reach, int* err, cudaStream_t s) {
  if (img_stride != (size_t)R * C)
    return set_error(ctx, WDL_ERR_UNSUPPORTED, "factor-resident axis pass: images must be contiguous");
  const size_t max_imgs = ((size_t)1 << 30) / ((size_t)R + 1);  // keep tile indices in int
  size_t done = 0;
  while (done < nimg) {
    size_t chunk = nimg - done;
    if (chunk > max_imgs) chunk = max_imgs;
    const float* src = in + done * img_stride;
    CUtensorMap tmap;
    const cuuint64_t dims[2] = {(cuuint64_t)C, (cuuint64_t)chunk * (cuuint64_t)R};
    const cuuint64_t strides[1] = {(cuuint64_t)C * sizeof(float)};
    const cuuint32_t box[2] = {(cuuint32_t)kAxKc, (cuuint32_t)kPxTR};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult cr = encode_tiled()(&tmap, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(src), dims,
                                       strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                       CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                                       CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (cr != CUDA_SUCCESS) return set_error(ctx, WDL_ERR_CUDA, "cuTensorMapEncodeTiled failed");
    const int nslab = (C + kAxTile - 1) / kAxTile;
    const long long tiles = (long long)chunk * ((R + kPxTR - 1) / kPxTR);
    long long per = ctx->sm_count / nslab;
    if (per < 1) per = 1;
    if (per > tiles) per = tiles;
    dim3 grid((unsigned)nslab, (unsigned)per);
    if (ctx->precision == WDL_SPLIT_BF16)
      tc_axis_persist_kernel<true><<<grid, kAxThreads, PxGeom::kSmem, s>>>(tmap, out + done * img_stride, G, R, C,
                                                                          (int)chunk, img_stride, reach, err);
    else
      tc_axis_persist_kernel<false><<<grid, kAxThreads, PxGeom::kSmem, s>>>(tmap, out + done * img_stride, G, R, C,
                                                                           (int)chunk, img_stride, reach, err);
    WDL_LAUNCH_CHECK(ctx);
    done += chunk;
  }
  return WDL_OK;
}

template <int TR>
int tc_axis_launch(wdl_ctx* ctx, const float* in, float* out, const uint8_t* G, int R, int C, size_t nimg,
                   size_t img_stride, int reach, int* err, cudaStream_t s) {
  size_t done = 0;
  while (done < nimg) {
    size_t chunk = nimg - done;
    if (chunk > 65535) chunk = 65535;
    dim3 grid((C + kAxTile - 1) / kAxTile, (R + TR - 1) / TR, (unsigned)chunk);
    const size_t smem = AxGeom<TR>::kSmem;
    if (ctx->precision == WDL_SPLIT_BF16)
      tc_axis_kernel<true, TR><<<grid, kAxThreads, smem, s>>>(in + done * img_stride, out + done * img_stride,
                                                              G, R, C, img_stride, reach, err);
    else
      tc_axis_kernel<false, TR><<<grid, kAxThreads, smem, s>>>(in + done * img_stride, out + done * img_stride,
                                                               G, R, C, img_stride, reach, err);
    WDL_LAUNCH_CHECK(ctx);
    done += chunk;
  }
  return WDL_OK;
}

// choice: the output tile height (64 or 128), plus 1000 for the copy-engine
// form; 2064 the persistent factor-resident form
int tc_axis_dispatch(wdl_ctx* ctx, int TR, const float* in, float* out, const uint8_t* G, int R, int C,
                     size_t nimg, size_t img_stride, int reach, int* err, cudaStream_t s) {
  if (TR == 2064) {
    if (tc_axis_persist_ok(in, C, reach) && img_stride == (size_t)R * C)
      return tc_axis_persist_launch(ctx, in, out, G, R, C, nimg, img_stride, reach, err, s);
    TR = 64;  // an unaligned call of a tuned shape: the same tile from the CTA's loads
  }
  if (TR >= 1000) {
    if (tc_axis_tma_ok(in, C))
      return TR == 1064 ? tc_axis_tma_launch<64>(ctx, in, out, G, R, C, nimg, img_stride, reach, err, s)
                        : tc_axis_tma_launch<128>(ctx, in, out, G, R, C, nimg, img_stride, reach, err, s);
    TR -= 1000;  // an unaligned call of a tuned shape: the same tile from the CTA's loads
  }
  return TR == 64 ? tc_axis_launch<64>(ctx, in, out, G, R, C, nimg, img_stride, reach, err, s)
                  : tc_axis_launch<128>(ctx, in, out, G, R, C, nimg, img_stride, reach, err, s);
}

// Default tile height: 64 while the 128-row grid would fill fewer than two
// waves of one CTA per SM (more, smaller tiles, two per SM), else 128.
int tc_axis_default_height(const wdl_ctx* ctx, int R, int C, size_t nimg) {
  const size_t tiles128 = (size_t)((C + kAxTile - 1) / kAxTile) * (size_t)((R + kAxTile - 1) / kAxTile) * nimg;
  return tiles128 < 2 * (size_t)ctx->sm_count ? 64 : 128;
}

// Tile height per shape (rows, row length, image count, precision): the first
// call of a shape outside a graph capture and outside profiling runs both
// heights on the call's own data (once untimed, once timed with CUDA events on
// the call's stream) and keeps the faster; with autotuning off (WDL_AUTOTUNE=0,
// wdl_set_autotune) the default height is taken.  Both heights issue the same
// MMAs for every output element (same K chunks, same order), so the choice
// does not change results.
int tc_axis_pass(wdl_ctx* ctx, const float* in, float* out, const uint8_t* G, int R, int C, size_t nimg,
                 size_t img_stride, int reach, int* err, cudaStream_t s) {
  const long long key[6] = {2, R, C, (long long)nimg, ctx->precision == WDL_SPLIT_BF16 ? 2 : 4, 0};
  for (const auto& e : ctx->tuned)
    if (!std::memcmp(e.key, key, sizeof(key)))
      return tc_axis_dispatch(ctx, e.choice, in, out, G, R, C, nimg, img_stride, reach, err, s);
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  cudaStreamIsCapturing(s, &cap);
  const int dflt = tc_axis_default_height(ctx, R, C, nimg);
  if (!autotune_enabled() || !ctx->autotune || cap != cudaStreamCaptureStatusNone || ctx->profiling)
    return tc_axis_dispatch(ctx, dflt, in, out, G, R, C, nimg, img_stride, reach, err, s);
  int cand_all[5] = {128, 64, 0, 0, 0};
  int ncand = 2;
  if (tc_axis_tma_ok(in, C) && img_stride == (size_t)R * C) {
    cand_all[ncand++] = 1128;
    cand_all[ncand++] = 1064;
    if (tc_axis_persist_ok(in, C, reach)) cand_all[ncand++] = 2064;
  }
  int best = dflt;
  float best_ms = 1e30f;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  WDL_CUDA_TRY(ctx, cudaEventCreate(&e0));
  WDL_CUDA_TRY(ctx, cudaEventCreate(&e1));
  int rc = WDL_OK;
  for (int ci = 0; ci < ncand; ++ci) {
    const int c = cand_all[ci];
    if ((rc = tc_axis_dispatch(ctx, c, in, out, G, R, C, nimg, img_stride, reach, err, s))) break;
    cudaEventRecord(e0, s);
    if ((rc = tc_axis_dispatch(ctx, c, in, out, G, R, C, nimg, img_stride, reach, err, s))) break;
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
  wdl_ctx::TuneEntry te;
  std::memcpy(te.key, key, sizeof(key));
  te.choice = best;
  te.ms = best_ms;
  ctx->tuned.push_back(te);
  return WDL_OK;
}

}  // namespace

size_t factor_block_bytes(int C) {
  const size_t nm = (C + kAxTile - 1) / kAxTile, nch = (C + kAxKc - 1) / kAxKc;
  return nm * nch * kAxOperand;
}

// Sets the kernels' SMEM limit and builds the factor blocks of every axis
// (blocks[a], at most 4 x 8 x 32 KB = 1 MB per axis for sides up to 512).
int tc_axis_init(wdl_ctx* ctx, uint8_t* (&blocks)[3]) {
  WDL_CUDA_TRY(ctx, cudaFuncSetAttribute(tc_axis_kernel<true, 128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)AxGeom<128>::kSmem));
  WDL_CUDA_TRY(ctx, cudaFuncSetAttribute(tc_axis_kernel<false, 128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)AxGeom<128>::kSmem));
  WDL_CUDA_TRY(ctx, cudaFuncSetAttribute(tc_axis_kernel<true, 64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)AxGeom<64>::kSmem));
  WDL_CUDA_TRY(ctx, cudaFuncSetAttribute(tc_axis_kernel<false, 64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)AxGeom<64>::kSmem));
  WDL_CUDA_TRY(ctx, cudaFuncSetAttribute(tc_axis_persist_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)PxGeom::kSmem));
  WDL_CUDA_TRY(ctx, cudaFuncSetAttribute(tc_axis_persist_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)PxGeom::kSmem));
  WDL_CUDA_TRY(ctx, cudaFuncSetAttribute(tc_axis_tma_kernel<true, 128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)AxTmaGeom<128>::kSmem));
  WDL_CUDA_TRY(ctx, cudaFuncSetAttribute(tc_axis_tma_kernel<false, 128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)AxTmaGeom<128>::kSmem));
  WDL_CUDA_TRY(ctx, cudaFuncSetAttribute(tc_axis_tma_kernel<true, 64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)AxTmaGeom<64>::kSmem));
  WDL_CUDA_TRY(ctx, cudaFuncSetAttribute(tc_axis_tma_kernel<false, 64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)AxTmaGeom<64>::kSmem));
  const bool split = ctx->precision == WDL_SPLIT_BF16;
  for (int a = 0; a < ctx->ndim; ++a) {
    const int C = ctx->axis_len[a];
    WDL_CUDA_TRY(ctx, cudaMalloc(&blocks[a], factor_block_bytes(C)));
    const unsigned nb = (unsigned)(factor_block_bytes(C) / kAxOperand);
    if (split) k_build_factor_blocks<true><<<nb, 256, 0, ctx->stream>>>(ctx->G32[a], C, blocks[a]);
    else k_build_factor_blocks<false><<<nb, 256, 0, ctx->stream>>>(ctx->G32[a], C, blocks[a]);
    WDL_LAUNCH_CHECK(ctx);
  }
  WDL_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return WDL_OK;
}

// The operator as axis passes, as the CUDA-core form: 2-D x then y through
// tmp; 3-D x, y, z.
int conv_stack_tc_axes(wdl_ctx* ctx, const float* in, float* out, float* tmp, size_t nimg,
                       uint8_t* const (&blocks)[3], int* err, cudaStream_t s) {
  const int W = ctx->W, H = ctx->H, D = ctx->D;
  const size_t N = ctx->N;
  int rc;
  if (ctx->ndim == 2) {
    if ((rc = tc_axis_pass(ctx, in, tmp, blocks[0], H, W, nimg, N, ctx->axis_reach[0], err, s))) return rc;
    return tc_axis_pass(ctx, tmp, out, blocks[1], W, H, nimg, N, ctx->axis_reach[1], err, s);
  }
  if ((rc = tc_axis_pass(ctx, in, out, blocks[0], D * H, W, nimg, N, ctx->axis_reach[0], err, s))) return rc;
  if ((rc = tc_axis_pass(ctx, out, tmp, blocks[1], W * D, H, nimg, N, ctx->axis_reach[1], err, s))) return rc;
  return tc_axis_pass(ctx, tmp, out, blocks[2], H * W, D, nimg, N, ctx->axis_reach[2], err, s);
}

}  // namespace wdl
