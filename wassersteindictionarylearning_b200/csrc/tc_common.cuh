// Shared device helpers of the tcgen05 kernels: operand-tile layout, BF16/TF32
// staging, GEMM issue and warpgroup barriers.
//
// Operand tiles use the canonical 128-byte-swizzled K-major layout: a tile of
// 128 rows is split along K into 128-byte column blocks ("regions") of
// 128 rows x 128 B; in a region, row r's 16-byte chunk c sits at chunk
// position c ^ (r % 8), and the UMMA descriptor addresses 8-row groups 1024 B
// apart.  Split BF16 keeps two planes (hi, lo) of 32 KB; TF32 one plane of 64 KB.
#pragma once

#include <cuda_bf16.h>

#include "tc_ptx.cuh"
#include "wdl_internal.cuh"

namespace wdl {
namespace tc {

constexpr int kRows = 128;               // tile rows (TMEM lanes / max grid side)
constexpr int kRegionBytes = kRows * 128; // one 128-byte column block of a tile
constexpr uint32_t kTmemCols = 256;      // per image stream: D1 [0,128), D2 [128,256)
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

// D[128 x N] = A[128 x K] * B[N x K]^T with A in tensor memory (lane = row,
// K along the columns: BF16 pairs or TF32 values, hi and lo planes for split
// BF16) and B a K-major SMEM tile.
template <bool SPLIT>
__device__ __forceinline__ void issue_gemm_ta(uint32_t d_tmem, uint32_t a_hi, uint32_t a_lo, uint32_t b_tile,
                                              int K, int N) {
  using F = Fmt<SPLIT>;
  const uint32_t id = ptx::idesc(F::fmt, 128, (uint32_t)N);
  const int steps = K / F::kstep;
  for (int ks = 0; ks < steps; ++ks) {
    const uint32_t byte = (uint32_t)ks * 32u;
    const uint32_t off = (byte >> 7) * kRegionBytes + (byte & 127u);
    const uint64_t b = ptx::sw128_desc(b_tile + off);
    const uint32_t col = (uint32_t)ks * 8u;  // 16 BF16 or 8 TF32 values
    if (SPLIT) {
      const uint64_t blo = ptx::sw128_desc(b_tile + F::plane_bytes + off);
      ptx::mma_bf16_ta(d_tmem, a_hi + col, b, id, ks > 0 ? 1u : 0u);
      ptx::mma_bf16_ta(d_tmem, a_hi + col, blo, id, 1u);
      ptx::mma_bf16_ta(d_tmem, a_lo + col, b, id, 1u);
    } else {
      ptx::mma_tf32_ta(d_tmem, a_hi + col, b, id, ks > 0 ? 1u : 0u);
    }
  }
}

// D1 (FP32 accumulators, columns [c0, c0 + 16) of this thread's lane) ->
// the A operand of the next GEMM in tensor memory: BF16 hi / lo pairs at
// a_hi / a_lo + c0 / 2, or TF32 values at a_hi + c0.  Follow with
// ptx::tmem_st_wait() before the GEMM is issued.
template <bool SPLIT>
__device__ __forceinline__ void restage16_tmem(uint32_t a_hi, uint32_t a_lo, uint32_t lane_base, int c0,
                                               const float (&v)[16]) {
  if (SPLIT) {
    uint32_t hi[8], lo[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const __nv_bfloat162 h = __floats2bfloat162_rn(v[2 * q], v[2 * q + 1]);
      const float2 hf = __bfloat1622float2(h);
      const __nv_bfloat162 l = __floats2bfloat162_rn(v[2 * q] - hf.x, v[2 * q + 1] - hf.y);
      hi[q] = *reinterpret_cast<const uint32_t*>(&h);
      lo[q] = *reinterpret_cast<const uint32_t*>(&l);
    }
    ptx::tmem_st8(a_hi + lane_base + (uint32_t)(c0 >> 1), hi);
    ptx::tmem_st8(a_lo + lane_base + (uint32_t)(c0 >> 1), lo);
  } else {
    uint32_t r[16];
#pragma unroll
    for (int q = 0; q < 16; ++q) r[q] = to_tf32(v[q]);
    ptx::tmem_st16(a_hi + lane_base + (uint32_t)c0, r);
  }
}

// Warpgroup-wide AND of a predicate (named barrier 1 + wg, 128 threads): keeps
// the control flow of a warpgroup uniform after bounded waits.
__device__ __forceinline__ bool wg_all(bool v, int wg) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 p, %1, 0;\n\t"
      "bar.red.and.pred q, %2, 128, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}\n"
      : "=r"(r)
      : "r"((uint32_t)v), "r"(1 + wg)
      : "memory");
  return r != 0;
}
__device__ __forceinline__ void wg_sync(int wg) {
  asm volatile("bar.sync %0, 128;" ::"r"(1 + wg) : "memory");
}
// Same for a stream of nthreads threads (named barrier 1 + id).
__device__ __forceinline__ bool bar_all(bool v, int id, int nthreads) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 p, %1, 0;\n\t"
      "bar.red.and.pred q, %2, %3, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}\n"
      : "=r"(r)
      : "r"((uint32_t)v), "r"(1 + id), "r"(nthreads)
      : "memory");
  return r != 0;
}
__device__ __forceinline__ void bar_sync(int id, int nthreads) {
  asm volatile("bar.sync %0, %1;" ::"r"(1 + id), "r"(nthreads) : "memory");
}

// Split 8 values into BF16 hi/lo 16-byte chunks, or 4 values into a TF32 chunk,
// and store them at (r, k0) (k0 a multiple of the chunk's element count).
template <bool SPLIT>
__device__ __forceinline__ void put_chunk(uint8_t* tile, int r, int k0, const float* v) {
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
    const uint32_t o = swz(r, k0, 2);
    *reinterpret_cast<uint4*>(tile + o) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
    *reinterpret_cast<uint4*>(tile + Fmt<true>::plane_bytes + o) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
  } else {
    *reinterpret_cast<uint4*>(tile + swz(r, k0, 4)) =
        make_uint4(to_tf32(v[0]), to_tf32(v[1]), to_tf32(v[2]), to_tf32(v[3]));
  }
}

// Resident factor tile: G[r][k] = g(|r-k|) for r, k < Gn, zero elsewhere.
template <bool SPLIT>
__device__ __forceinline__ void load_factor(uint8_t* g_tile, const float* __restrict__ G, int Gn,
                                            int t, int nthreads) {
  for (int e = t; e < kRows * kRows; e += nthreads) {
    const int r = e >> 7, k = e & 127;
    const float v = (r < Gn && k < Gn) ? G[(size_t)r * Gn + k] : 0.f;
    put1<SPLIT>(g_tile, r, k, v);
  }
}

}  // namespace tc
}  // namespace wdl
