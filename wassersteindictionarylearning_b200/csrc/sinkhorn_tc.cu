// Persistent, dependency-driven tensor-core kernel for the whole Sinkhorn
// forward pass, loss and reverse pass of P histograms (grid sides <= 128,
// kernel domain, TF32 or split-BF16 operators, FP32 scalings and tape).
//
// Work items, claimed in order from one atomic counter by 2 warpgroups per CTA:
//   FWD (it, p, k), it = 1..L          (cpp/inverseWasserstein.h:565-593)
//     X1 = b[it-1] = bary[it-1]/phi[it-1] (b[0] = ones or the warm start)
//     cb = G*X1 (stored), X2 = p_k/cb, phi[it] = G*X2 (stored)
//   DICT (s, p, k), s = L..1           (:602-629)
//     X1 = (lambda n - v) * b[s]; c = G*X1; gdic += c/cb[s-1];
//     X2 = -p c/cb[s-1]^2; v = (G*X2)/phi[s-1]          (s = 1 stops after gdic)
//   WGT (s, p, k), s = L..1            (:635-673)
//     dot += sum log(phi[s]) gw;  X1 = (lambda gw - r)/phi[s];
//     X2 = (G*X1)(-p/cb[s-1]^2); r = (G*X2) b[s-1]       (s = 1 stops after dot)
// The cross-atom reductions are accumulated by the producing epilogues with
// vector red.global.add into L2-resident buffers: FWD adds lambda_k
// safe_log(phi_k) into acc[it][p] (bary[it] = exp(acc)), DICT adds v into
// n[p] and WGT adds r into gw[p] (double-buffered by step parity).  An atomic
// count per histogram detects the item that completes a group; it publishes a
// per-histogram release flag (after the last forward iteration it also forms
// the loss and the reverse-pass start n = g, gw = g*bary; in the reverse pass
// it clears the message buffer the next step accumulates into).  Consumers wait
// on the flags with a bounded acquire spin; an item only waits on items claimed
// before it, so progress never depends on all CTAs being resident.  The float
// atomics make the summation order of the K terms run-dependent (results are
// reproducible to FP32 rounding, not bitwise).
//
// Each item runs two separable convolutions.  The first is in "column form"
// (TMEM lane = x: the operand is staged from row-major global data and the
// result is read back as columns), the second in "row form" (lane = y): the
// column-form result, after the elementwise step, is exactly the row form's
// K-major operand, so every SMEM write is a whole 16-byte chunk and every
// global access of the epilogue is a contiguous row segment.
#include <cfloat>

#include "tc_common.cuh"
#include "wdl_math.cuh"

namespace wdl {

namespace {
using namespace tc;

constexpr uint64_t kDepWaitNs = 4000000000ull;  // default bound on a dependency wait

__device__ __forceinline__ int ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(int* p, int v) {
  asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ bool wait_ge(const int* flag, int target, uint64_t limit_ns) {
  if (ld_acquire(flag) >= target) return true;
  const uint64_t t0 = ptx::globaltimer_ns();
  while (true) {
    __nanosleep(100);
    if (ld_acquire(flag) >= target) return true;
    if (ptx::globaltimer_ns() - t0 > limit_ns) return false;
  }
}



constexpr int kSt = 256;   // threads of one image stream (8 warps)
constexpr int kWarps = kSt / 32;

// Fast intrinsics for the tensor-core precisions: the operators themselves
// round to TF32 or split BF16, so the elementwise steps use the hardware
// reciprocal, exp2 and log2 (relative error ~1e-7, far below the operator's).
__device__ __forceinline__ float fdiv(float a, float b) { return __fdividef(a, b); }
__device__ __forceinline__ float frcp(float b) { return __fdividef(1.0f, b); }

// Stream-wide sum of a double (result valid in every thread of the stream).
__device__ __forceinline__ double st_sum(double v, double* scratch, int st, int t) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((t & 31) == 0) scratch[st * kWarps + (t >> 5)] = v;
  bar_sync(st, kSt);
  double tot = 0;
#pragma unroll
  for (int w = 0; w < kWarps; ++w) tot += scratch[st * kWarps + w];
  bar_sync(st, kSt);
  return tot;
}

// Pulls an image into L2 ahead of use with one bulk prefetch by the copy
// engine (its 16-byte aligned interior), issued by one thread: no registers,
// no wait, and no load-unit traffic in the issuing stream (thread-issued
// per-line prefetches cost the reverse items ~1.4 us of issue each).
__device__ __forceinline__ void prefetch_l2(const float* p, size_t n, int t) {
  if (t == 0) {
    const uintptr_t a0 = (reinterpret_cast<uintptr_t>(p) + 15) & ~uintptr_t(15);
    const uintptr_t a1 = (reinterpret_cast<uintptr_t>(p + n)) & ~uintptr_t(15);
    if (a1 > a0)
      asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a0), "r"((uint32_t)(a1 - a0)) : "memory");
  }
}

// Phase trace (thread 0 of a stream; only when a trace buffer is given):
// claim, dependency wait, prologue, first convolution, mid, second
// convolution, epilogue, completion; slot 8 counts items.
struct Trace {
  unsigned long long* buf;
  uint64_t last;
  int type;
  __device__ void start(unsigned long long* b, int t0) {
    buf = t0 == 0 ? b : nullptr;
    if (buf) last = ptx::globaltimer_ns();
  }
  __device__ void mark(int phase) {
    if (!buf) return;
    const uint64_t now = ptx::globaltimer_ns();
    atomicAdd(&buf[type * 9 + phase], (unsigned long long)(now - last));
    last = now;
  }
};

struct Geo {
  int W, H, Wp, Hp;
  uint32_t cpr, cpr_magic;  // operand chunks per row, ceil(2^32 / cpr)
  bool vec;
};

template <int NIN, int CE, int A>
__device__ __forceinline__ void load_row_chunk(float (&in)[NIN > 0 ? NIN : 1][CE],
                                               const float* const (&src)[NIN > 0 ? NIN : 1], int i, int x0,
                                               bool row_ok, const Geo& g) {
  if constexpr (A < NIN) {
    const float* row = src[A] + (size_t)i * g.W;
    if (row_ok && g.vec && x0 + CE <= g.W) {
#pragma unroll
      for (int q = 0; q < CE; q += 4) {
        const float4 f4 = __ldcg(reinterpret_cast<const float4*>(row + x0 + q));
        in[A][q] = f4.x; in[A][q + 1] = f4.y; in[A][q + 2] = f4.z; in[A][q + 3] = f4.w;
      }
    } else {
#pragma unroll
      for (int q = 0; q < CE; ++q) in[A][q] = (row_ok && x0 + q < g.W) ? __ldcg(row + x0 + q) : 0.f;
    }
    load_row_chunk<NIN, CE, A + 1>(in, src, i, x0, row_ok, g);
  }
}

// Stage the column-form operand X1(i, x) = f(in_0..in_{NIN-1} at (i, x)) for
// rows i < Hp, x < Wp (zero outside the H x W image).  UNR chunks of loads are
// issued before any is consumed.  f may accumulate side sums (captured by
// reference); it is only called for pixels inside the image.
template <bool SPLIT, int NIN, class F>
__device__ __forceinline__ void stage_rows(uint8_t* tile, const float* const (&src)[NIN > 0 ? NIN : 1],
                                           F f, const Geo& g, int t) {
  constexpr int CE = SPLIT ? 8 : 4;
  constexpr int UNR = NIN > 2 ? 1 : 2;
  const int total = g.Hp * (int)g.cpr;
  for (int base = t; base < total; base += kSt * UNR) {
    float in[UNR][NIN > 0 ? NIN : 1][CE];
    int iu[UNR], xu[UNR];
#pragma unroll
    for (int u = 0; u < UNR; ++u) {
      const int c = base + u * kSt;
      const int i = (int)__umulhi((uint32_t)c, g.cpr_magic);
      const int x0 = (c - i * (int)g.cpr) * CE;
      iu[u] = i;
      xu[u] = x0;
      const bool row_ok = c < total && i < g.H;
      load_row_chunk<NIN, CE, 0>(in[u], src, i, x0, row_ok, g);
    }
#pragma unroll
    for (int u = 0; u < UNR; ++u) {
      if (base + u * kSt >= total) break;
      const int i = iu[u], x0 = xu[u];
      float out[CE];
#pragma unroll
      for (int q = 0; q < CE; ++q) {
        float av[NIN > 0 ? NIN : 1];
#pragma unroll
        for (int s = 0; s < NIN; ++s) av[s] = in[u][s][q];
        out[q] = (i < g.H && x0 + q < g.W) ? f(av) : 0.f;
      }
      put_chunk<SPLIT>(tile, i, x0, out);
    }
  }
}

struct Ctl {
  uint8_t* tile;
  uint32_t g_a, x_a, bar_a, d1, d2, a_hi, a_lo, lane_base;
  int st, t, lane_row, half;
  uint32_t phase;
};

// Separable convolution of the operand tile: MMA1 (A = G, B = tile rows n, K =
// K1) -> D1 -> restaged in tensor memory as the A operand (row = this thread's
// lane; warps w and w+4 of the stream take alternate 16-column chunks of the
// same lanes) -> MMA2 (A from tensor memory, B = G) -> D2 in D1's columns.
// Column form: K1 = Wp, N1 = Hp; row form: K1 = Hp, N1 = Wp.
template <bool SPLIT>
__device__ bool gemm_pair(Ctl& c, int K1, int N1) {
  ptx::tc_fence_before();
  ptx::fence_proxy_async_smem();
  bar_sync(c.st, kSt);
  if (c.t == 0) {
    ptx::tc_fence_after();
    issue_gemm<SPLIT>(c.d1, c.g_a, c.x_a, K1, N1);
    ptx::mma_commit(c.bar_a);
  }
  bool ok = bar_all(ptx::mbar_wait(c.bar_a, c.phase, kWaitNs), c.st, kSt);
  c.phase ^= 1;
  ptx::tc_fence_after();
  // D1 -> the second GEMM's A operand, kept in tensor memory (split into BF16
  // hi / lo, or rounded to TF32); the second GEMM then overwrites D1's columns
  for (int c0 = 16 * c.half; c0 < N1; c0 += 32) {
    float v[16];
    ptx::tmem_ld16(c.d1 + c.lane_base + (uint32_t)c0, v);
    ptx::tmem_ld_wait();
    restage16_tmem<SPLIT>(c.a_hi, c.a_lo, c.lane_base, c0, v);
  }
  ptx::tmem_st_wait();
  ptx::tc_fence_before();
  bar_sync(c.st, kSt);
  if (c.t == 0) {
    ptx::tc_fence_after();
    issue_gemm_ta<SPLIT>(c.d2, c.a_hi, c.a_lo, c.g_a, N1, N1);
    ptx::mma_commit(c.bar_a);
  }
  ok = bar_all(ok && ptx::mbar_wait(c.bar_a, c.phase, kWaitNs), c.st, kSt);
  c.phase ^= 1;
  ptx::tc_fence_after();
  return ok;
}

// Column-form result D2[x][i] (x = this thread's lane): Y(i, x) for rows i in
// chunks of 16.  For each chunk the NIN inputs at the 16 pixels idx = i*W + x
// are loaded first (all loads in flight together), then m(idx, y, in) consumes
// them (it may store) and returns the next operand's value, written as row x
// (K = i) of the tile when stage_next.
template <int NIN, int A>
__device__ __forceinline__ void load_col_chunk(float (&in)[NIN][16], const float* const (&src)[NIN], int c0,
                                               int x, const Geo& g) {
  if constexpr (A < NIN) {
#pragma unroll
    for (int t = 0; t < 16; ++t) {
      const int i = c0 + t;
      in[A][t] = (x < g.W && i < g.H) ? __ldcg(src[A] + (size_t)i * g.W + x) : 1.f;
    }
    load_col_chunk<NIN, A + 1>(in, src, c0, x, g);
  }
}

template <bool SPLIT, int NIN, class M>
__device__ __forceinline__ void mid_columns(Ctl& c, const Geo& g, const float* const (&src)[NIN], M m,
                                            bool stage_next) {
  const int x = c.lane_row;
  for (int c0 = 16 * c.half; c0 < g.Hp; c0 += 32) {
    float in[NIN][16];
    load_col_chunk<NIN, 0>(in, src, c0, x, g);
    float y[16];
    ptx::tmem_ld16(c.d2 + c.lane_base + (uint32_t)c0, y);
    ptx::tmem_ld_wait();
#pragma unroll
    for (int t = 0; t < 16; ++t) {
      const int i = c0 + t;
      float iv[NIN];
#pragma unroll
      for (int q = 0; q < NIN; ++q) iv[q] = in[q][t];
      y[t] = (x < g.W && i < g.H) ? m((size_t)i * g.W + x, y[t], iv) : 0.f;
    }
    if (stage_next) put16<SPLIT>(c.tile, x, c0, y);
  }
}

template <int NIN, int A>
__device__ __forceinline__ void load_px4(float (&in)[NIN > 0 ? NIN : 1][4], const float* const (&src)[NIN > 0 ? NIN : 1],
                                         size_t idx, bool okr, int x0, const Geo& g) {
  if constexpr (A < NIN) {
    if (okr && g.vec) {
      const float4 f = __ldcg(reinterpret_cast<const float4*>(src[A] + idx));
      in[A][0] = f.x; in[A][1] = f.y; in[A][2] = f.z; in[A][3] = f.w;
    } else {
#pragma unroll
      for (int r = 0; r < 4; ++r) in[A][r] = (okr && x0 + r < g.W) ? __ldcg(src[A] + idx + r) : 1.f;
    }
    load_px4<NIN, A + 1>(in, src, idx, okr, x0, g);
  }
}

__device__ __forceinline__ void red_add4(float* p, float a, float b, float c, float d) {
  asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(p), "f"(a), "f"(b), "f"(c), "f"(d) : "memory");
}
__device__ __forceinline__ float safe_logf(float x) { return x > 0.f ? __logf(x) : (float)kLogEpsilon; }

// Row-form result D2[i][x] (i = this thread's lane) with an accumulating
// epilogue.  The result is first staged in the (now free) operand tile as a
// row-major FP32 image (512-byte rows, 16-byte chunk j of row i at position
// j ^ (i % 8)), then the stream walks it row by row: 32 threads x 16 bytes
// cover one row, so every global load, store and red is a contiguous 512-byte
// row.  e(idx, y4, in4) gets 4 consecutive pixels, may store, and returns the
// 4 values added into acc[idx..idx+3].
template <int NIN, class E>
__device__ __forceinline__ void epi_rows_red(Ctl& c, const Geo& g, const float* const (&src)[NIN > 0 ? NIN : 1],
                                             float* acc, E e) {
  {
    const int i = c.lane_row;
    uint8_t* rowp = c.tile + (size_t)i * 512;
    for (int c0 = 16 * c.half; c0 < g.Wp; c0 += 32) {
      float y[16];
      ptx::tmem_ld16(c.d2 + c.lane_base + (uint32_t)c0, y);
      ptx::tmem_ld_wait();
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int j = (c0 >> 2) + q;
        *reinterpret_cast<float4*>(rowp + ((j ^ (i & 7)) << 4)) =
            make_float4(y[4 * q], y[4 * q + 1], y[4 * q + 2], y[4 * q + 3]);
      }
    }
  }
  bar_sync(c.st, kSt);
  const int j = c.t & 31;  // 16-byte chunk of the row
  const int x0 = 4 * j;
  constexpr int U = 2;
  for (int i0 = c.t >> 5; i0 < g.H; i0 += kWarps * U) {
    float4 y4[U];
    float in[U][NIN > 0 ? NIN : 1][4];
    int iu[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int i = i0 + u * kWarps;
      iu[u] = i;
      const bool okr = i < g.H && x0 < g.W;
      y4[u] = okr ? *reinterpret_cast<const float4*>(c.tile + (size_t)i * 512 + ((j ^ (i & 7)) << 4))
                  : make_float4(0.f, 0.f, 0.f, 0.f);
      const size_t idx = (size_t)i * g.W + x0;
      load_px4<NIN, 0>(in[u], src, idx, okr, x0, g);
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int i = iu[u];
      if (i >= g.H || x0 >= g.W) continue;
      const size_t idx = (size_t)i * g.W + x0;
      const int nv = g.W - x0 < 4 ? g.W - x0 : 4;
      const float4 out = e(idx, y4[u], in[u], nv);
      if (g.vec) {
        red_add4(acc + idx, out.x, out.y, out.z, out.w);
      } else {
        const float o[4] = {out.x, out.y, out.z, out.w};
        for (int r = 0; r < nv; ++r) atomicAdd(acc + idx + r, o[r]);
      }
    }
  }
}

// Stores 4 consecutive values (nv valid; 16-byte store when the row is aligned).
__device__ __forceinline__ void st4(float* p, float4 v, int nv, bool vec) {
  if (vec) {
    __stcg(reinterpret_cast<float4*>(p), v);
  } else {
    const float o[4] = {v.x, v.y, v.z, v.w};
    for (int r = 0; r < nv; ++r) __stcg(p + r, o[r]);
  }
}

template <bool SPLIT>
__global__ void __launch_bounds__(2 * kSt, 1) sinkhorn_tc_kernel(const SkArgs a) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* base = reinterpret_cast<uint8_t*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int st = warp / kWarps, t = tid % kSt, ws = warp % kWarps;
  uint8_t* g_tile = base;
  uint64_t* bars = reinterpret_cast<uint64_t*>(base + 3 * kTileBytes);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(base + 3 * kTileBytes + 16);
  int* s_int = reinterpret_cast<int*>(base + 3 * kTileBytes + 32);          // [2][4]
  double* s_dbl = reinterpret_cast<double*>(base + 3 * kTileBytes + 64);    // [2][kWarps]
  SkProblem* s_prob = reinterpret_cast<SkProblem*>(base + 3 * kTileBytes + 256);  // [2]

  load_factor<SPLIT>(g_tile, a.G, a.Gn, tid, blockDim.x);
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

  Ctl c;
  c.tile = base + (1 + st) * kTileBytes;
  c.g_a = ptx::smem_addr(g_tile);
  c.x_a = ptx::smem_addr(c.tile);
  c.bar_a = ptx::smem_addr(&bars[st]);
  // per stream: D1 and D2 share columns [0, 128), the second GEMM's A operand
  // in tensor memory takes [128, 256) (BF16 hi [128, 192), lo [192, 256))
  c.d1 = *tmem_slot + (uint32_t)st * kTmemCols;
  c.d2 = c.d1;
  c.a_hi = c.d1 + 128;
  c.a_lo = c.d1 + 192;
  c.lane_base = (uint32_t)((ws & 3) * 32) << 16;
  c.st = st;
  c.t = t;
  c.lane_row = (ws & 3) * 32 + lane;
  c.half = ws >> 2;
  c.phase = 0;

  int* work = a.sync;
  int* err = a.sync + 1;
  SkProblem* const pr = &s_prob[st];
  int cur_q = -1;
  Trace tr;
  while (true) {
    tr.start(a.trace, t);
    tr.type = 0;
    if (t == 0) {
      const int item = atomicAdd(work, 1);
      int q = 0, type = 0, step = 0, pkv = 0;
      if (item < a.total) {
        if (a.items) {
          const int4 d = a.items[item];
          q = d.x; type = d.y; step = d.z; pkv = d.w;
        } else {  // one problem: forward items, then per reverse step its items
          const SkProblem& p0 = a.probs[0];
          const long long PK = (long long)p0.P * p0.K;
          if (item < (long long)p0.L * PK) {
            type = 0;
            step = (int)(item / PK) + 1;
            pkv = (int)(item % PK);
          } else {
            const long long per = p0.need_dic ? 2 * PK : PK;
            const long long j = item - (long long)p0.L * PK;
            step = p0.L - (int)(j / per);
            const long long rem = j % per;
            pkv = (int)(p0.need_dic ? rem >> 1 : rem);
            type = p0.need_dic ? 1 + (int)(rem & 1) : 2;
          }
        }
      }
      s_int[st * 4] = item < a.total ? q : -1;
      s_int[st * 4 + 1] = type;
      s_int[st * 4 + 2] = step;
      s_int[st * 4 + 3] = pkv;
    }
    bar_sync(st, kSt);
    const int q = s_int[st * 4];
    if (q < 0) break;
    const int type = s_int[st * 4 + 1], step = s_int[st * 4 + 2];
    const long long pk = s_int[st * 4 + 3];
    if (q != cur_q) {  // this stream's problem descriptor, staged in SMEM
      const int nw = (int)(sizeof(SkProblem) / 4);
      if (t < nw) reinterpret_cast<uint32_t*>(pr)[t] = reinterpret_cast<const uint32_t*>(&a.probs[q])[t];
      cur_q = q;
    }
    bar_sync(st, kSt);
    tr.type = type;
    const int K = pr->K, L = pr->L, P = pr->P;
    const size_t N = pr->N, PN = (size_t)P * N, PKN = (size_t)P * K * N;
    const int p = (int)(pk / K), k = (int)(pk % K);
    Geo g;
    g.W = pr->W;
    g.H = pr->H;
    g.Wp = pr->Wp;
    g.Hp = pr->Hp;
    g.cpr = pr->cpr;
    g.cpr_magic = pr->cpr_magic;
    g.vec = pr->vec != 0;
    const bool fwd_only = pr->fwd_only != 0;
    int* done_fwd = pr->sync;
    int* bary_ready = done_fwd + P;
    int* done_bwd = bary_ready + P;
    int* msg_ready = done_bwd + P;
    int* range = msg_ready + P;  // a scaling of histogram p left the FP32 range
    // Tape slot of iteration it (1..L): all L kept for the reverse pass; two
    // slots suffice for a forward-only run.
    auto slot = [&](int it) -> size_t { return fwd_only ? (size_t)((it - 1) & 1) : (size_t)(it - 1); };
    {  // every array this item reads, requested into L2 up front
      const size_t pkN = (size_t)pk * N, pN = (size_t)p * N;
      if (type == 0) {
        if (step > 1) {
          prefetch_l2(pr->acc + slot(step - 1) * PN + pN, N, t);
          prefetch_l2(pr->phi + slot(step - 1) * PKN + pkN, N, t);
        } else if (pr->b0) {
          prefetch_l2(pr->b0 + pkN, N, t);
        }
      } else {
        const int s = step;
        prefetch_l2(pr->phi + slot(s) * PKN + pkN, N, t);
        prefetch_l2(pr->cb + slot(s) * PKN + pkN, N, t);
        if (s > 1) prefetch_l2(pr->phi + slot(s - 1) * PKN + pkN, N, t);
        if (type == 1) {
          prefetch_l2(pr->nb + (size_t)(s & 1) * PN + pN, N, t);
          prefetch_l2(pr->v + pkN, N, t);
          prefetch_l2(pr->acc + slot(s) * PN + pN, N, t);
          prefetch_l2(pr->gdic + pkN, N, t);
        } else {
          prefetch_l2(pr->gwb + (size_t)(s & 1) * PN + pN, N, t);
          prefetch_l2(pr->r + pkN, N, t);
          if (s > 1) prefetch_l2(pr->acc + slot(s - 1) * PN + pN, N, t);
        }
      }
    }
    tr.mark(0);
    if (t == 0) {
      bool ok = true;
      if (type == 0) {
        if (step > 1) ok = wait_ge(&bary_ready[p], step - 1, a.dep_wait_ns);
      } else {
        ok = wait_ge(&msg_ready[p], L - step, a.dep_wait_ns);
      }
      s_int[st * 4 + 1] = ok ? 1 : 0;
    }
    bar_sync(st, kSt);
    if (!s_int[st * 4 + 1]) {
      if (t == 0) atomicExch(err, WDL_ERR_TIMEOUT);
      break;
    }
    tr.mark(1);
    const float lam = pr->lam[pk];
    const float* atom = pr->atoms + (size_t)k * N;
    bool ok = true;

    if (type == 0) {  // ---------------- forward Bregman iteration
      const int it = step;
      // Scalings beyond the FP32 range (narrow kernels: they grow with the
      // iterations where FP64 still holds them) saturate to inf or to 0.  Every
      // such chain reaches phi = conv(a) as 0 (b = bary / phi overflows) or
      // inf (a = p / conv_b overflows): a histogram whose phi leaves (0, inf)
      // is flagged, and after the launch its barycenter, loss and gradients
      // are set to NaN (k_poison_flagged).
      bool bad = false;
      float* cb_out = pr->cb + slot(it) * PKN + pk * N;
      float* phi_out = pr->phi + slot(it) * PKN + pk * N;
      float* acc_out = pr->acc + slot(it) * PN + (size_t)p * N;
      if (it == 1) {
        if (pr->b0) {
          const float* src[1] = {pr->b0 + pk * N};
          stage_rows<SPLIT, 1>(c.tile, src, [](const float (&v)[1]) { return v[0]; }, g, t);
        } else {
          const float* src[1] = {atom};
          stage_rows<SPLIT, 0>(c.tile, src, [](const float (&)[1]) { return 1.f; }, g, t);
        }
      } else {  // b[it-1] = exp(acc[it-1]) / phi[it-1]
        const float* src[2] = {pr->acc + slot(it - 1) * PN + (size_t)p * N,
                               pr->phi + slot(it - 1) * PKN + pk * N};
        stage_rows<SPLIT, 2>(c.tile, src, [](const float (&v)[2]) { return fdiv(__expf(v[0]), v[1]); }, g, t);
      }
      tr.mark(2);
      const float* msrc[1] = {atom};
      ok = gemm_pair<SPLIT>(c, g.Wp, g.Hp);
      tr.mark(3);
      const bool keep_cb = !fwd_only;
      mid_columns<SPLIT, 1>(c, g, msrc, [&](size_t idx, float y, const float (&in)[1]) {
        if (keep_cb) __stcg(cb_out + idx, y);  // read again only in the reverse pass
        return fdiv(in[0], y);
      }, true);
      tr.mark(4);
      ok = ok && gemm_pair<SPLIT>(c, g.Hp, g.Wp);
      tr.mark(5);
      const float* esrc[1] = {nullptr};
      epi_rows_red<0>(c, g, esrc, acc_out, [&](size_t idx, float4 y, const float (&)[1][4], int nv) {
        st4(phi_out + idx, y, nv, g.vec);
        const float o[4] = {y.x, y.y, y.z, y.w};
        for (int r = 0; r < nv; ++r) bad |= !(o[r] > 0.f && o[r] <= FLT_MAX);
        return make_float4(lam * safe_logf(y.x), lam * safe_logf(y.y), lam * safe_logf(y.z),
                           lam * safe_logf(y.w));
      });
      if (bad) *(volatile int*)(range + p) = 1;
      tr.mark(6);
    } else if (type == 1) {  // ---------------- reverse pass, dictionary recursion
      const int s = step;
      const float* src[4] = {pr->nb + (size_t)(s & 1) * PN + (size_t)p * N, pr->v + pk * N,
                             pr->acc + slot(s) * PN + (size_t)p * N, pr->phi + slot(s) * PKN + pk * N};
      stage_rows<SPLIT, 4>(
          c.tile, src, [lam](const float (&v)[4]) { return (lam * v[0] - v[1]) * fdiv(__expf(v[2]), v[3]); }, g,
          t);
      tr.mark(2);
      const float* cbp = pr->cb + slot(s) * PKN + pk * N;  // cb[s-1] sits in slot(s)
      float* gd = pr->gdic + pk * N;
      const float* msrc[3] = {cbp, gd, atom};
      ok = gemm_pair<SPLIT>(c, g.Wp, g.Hp);
      tr.mark(3);
      mid_columns<SPLIT, 3>(c, g, msrc, [&](size_t idx, float y, const float (&in)[3]) {
        const float rc = frcp(in[0]);
        const float q2 = y * rc;
        __stcg(gd + idx, in[1] + q2);
        return -in[2] * q2 * rc;
      }, s > 1);
      tr.mark(4);
      if (s > 1) {
        const float* php = pr->phi + slot(s - 1) * PKN + pk * N;
        const float* esrc[1] = {php};
        ok = ok && gemm_pair<SPLIT>(c, g.Hp, g.Wp);
        tr.mark(5);
        float* vout = pr->v + pk * N;
        float* nout = pr->nb + (size_t)((s - 1) & 1) * PN + (size_t)p * N;
        epi_rows_red<1>(c, g, esrc, nout, [&](size_t idx, float4 y, const float (&in)[1][4], int nv) {
          const float4 vv = make_float4(fdiv(y.x, in[0][0]), fdiv(y.y, in[0][1]), fdiv(y.z, in[0][2]),
                                        fdiv(y.w, in[0][3]));
          st4(vout + idx, vv, nv, g.vec);
          return vv;
        });
        tr.mark(6);
      }
    } else {  // ---------------- reverse pass, weight recursion
      const int s = step;
      const float* src[3] = {pr->gwb + (size_t)(s & 1) * PN + (size_t)p * N, pr->r + pk * N,
                             pr->phi + slot(s) * PKN + pk * N};
      double dacc = 0;
      stage_rows<SPLIT, 3>(c.tile, src, [lam, &dacc](const float (&v)[3]) {
        dacc += (double)__logf(v[2]) * (double)v[0];
        return fdiv(lam * v[0] - v[1], v[2]);
      }, g, t);
      const double dsum = st_sum(dacc, s_dbl, st, t);
      if (t == 0) atomicAdd(&pr->dot[pk], dsum);
      tr.mark(2);
      if (s > 1) {
        const float* cbp = pr->cb + slot(s) * PKN + pk * N;
        const float* msrc[2] = {cbp, atom};
        ok = gemm_pair<SPLIT>(c, g.Wp, g.Hp);
        tr.mark(3);
        mid_columns<SPLIT, 2>(c, g, msrc, [&](size_t idx, float y, const float (&in)[2]) {
          const float rc = frcp(in[0]);
          return y * (-in[1] * rc * rc);
        }, true);
        tr.mark(4);
        const float* php = pr->phi + slot(s - 1) * PKN + pk * N;
        const float* accp = pr->acc + slot(s - 1) * PN + (size_t)p * N;
        const float* esrc[2] = {accp, php};
        ok = ok && gemm_pair<SPLIT>(c, g.Hp, g.Wp);
        tr.mark(5);
        float* rout = pr->r + pk * N;
        float* gout = pr->gwb + (size_t)((s - 1) & 1) * PN + (size_t)p * N;
        epi_rows_red<2>(c, g, esrc, gout, [&](size_t idx, float4 y, const float (&in)[2][4], int nv) {
          const float4 rr = make_float4(y.x * fdiv(__expf(in[0][0]), in[1][0]),
                                        y.y * fdiv(__expf(in[0][1]), in[1][1]),
                                        y.z * fdiv(__expf(in[0][2]), in[1][2]),
                                        y.w * fdiv(__expf(in[0][3]), in[1][3]));
          st4(rout + idx, rr, nv, g.vec);
          return rr;
        });
        tr.mark(6);
      }
    }
    if (!ok) {
      if (t == 0) atomicExch(err, WDL_ERR_TIMEOUT);
      break;
    }

    // Completion: the item that finishes a group publishes it.
    bar_sync(st, kSt);
    if (t == 0) {
      __threadfence();
      int fin;
      if (type == 0) fin = atomicAdd(&done_fwd[p], 1) + 1 == step * K;
      else fin = atomicAdd(&done_bwd[p], 1) + 1 == (pr->need_dic ? 2 : 1) * K * (L - step + 1);
      s_int[st * 4 + 2] = fin;
    }
    bar_sync(st, kSt);
    if (!s_int[st * 4 + 2]) {
      tr.mark(7);
      if (tr.buf) atomicAdd(&tr.buf[type * 9 + 8], 1ull);
      continue;
    }
    __threadfence();
    if (type == 0) {
      const int it = step;
      if (fwd_only && it >= 2) {
        // acc[it-1] has been read by every item of iteration it: clear its slot,
        // which iteration it+1 accumulates into.
        float* z = pr->acc + slot(it + 1) * PN + (size_t)p * N;
        for (size_t j = t; j < N; j += kSt) __stcg(z + j, 0.f);
      }
      const bool last = it == L && !fwd_only;
      if (last) {  // loss and its gradient (cpp/loss.h:19-90); messages for s = L
        const float* accL = pr->acc + slot(L) * PN + (size_t)p * N;
        float* n0 = pr->nb + (size_t)(L & 1) * PN + (size_t)p * N;
        float* g0 = pr->gwb + (size_t)(L & 1) * PN + (size_t)p * N;
        const bool dic = pr->need_dic != 0;
        const int lt = pr->loss_type;
        double lacc = 0;
        for (size_t j = t; j < N; j += kSt) {
          const float bv = expf(__ldcg(accL + j));
          const double o = pr->obs[(size_t)p * N + j];
          const float o32 = (float)o;
          float gg;
          if (lt == WDL_LOSS_TV) {
            lacc += fabs((double)bv - o);
            gg = (bv - o32) > 0.f ? 0.5f : -0.5f;
          } else if (lt == WDL_LOSS_QUADRATIC) {
            const double d = (double)bv - o;
            lacc += d * d;
            gg = 2.f * (bv - o32);
          } else {
            const double rr = (double)bv / o;
            lacc += (double)bv * log(rr > kEpsilon ? rr : kEpsilon) - (double)bv + o;
            const float q2 = bv / o32;
            gg = q2 > 0.f ? logf(q2) : (float)kLogEpsilon;
          }
          if (dic) __stcg(n0 + j, gg);
          __stcg(g0 + j, gg * bv);
        }
        const double tot = st_sum(lacc, s_dbl, st, t);
        if (t == 0) pr->loss[p] = lt == WDL_LOSS_TV ? 0.5 * tot : tot;
      }
      bar_sync(st, kSt);
      if (t == 0) {
        __threadfence();
        st_release(&bary_ready[p], it);
        if (last) st_release(&msg_ready[p], 0);
      }
    } else {
      const int s = step;
      if (s > 1) {  // the messages step s consumed are cleared for step s-2's sums
        float* zn = pr->nb + (size_t)(s & 1) * PN + (size_t)p * N;
        float* zg = pr->gwb + (size_t)(s & 1) * PN + (size_t)p * N;
        const bool dic = pr->need_dic != 0;
        for (size_t j = t; j < N; j += kSt) {
          if (dic) __stcg(zn + j, 0.f);
          __stcg(zg + j, 0.f);
        }
      }
      bar_sync(st, kSt);
      if (t == 0) {
        __threadfence();
        st_release(&msg_ready[p], L - s + 1);
      }
    }
    tr.mark(7);
    if (tr.buf) atomicAdd(&tr.buf[type * 9 + 8], 1ull);
  }
  __syncthreads();
  ptx::tc_fence_after();
  if (warp == 0) ptx::tmem_dealloc(*tmem_slot, 2 * kTmemCols);
}

// Histograms whose forward pass flagged scalings beyond the FP32 range
// (range[p]): barycenter, loss, weight gradient and their share of the
// dictionary gradient set to NaN, as an overflow in FP64 would leave them.
__global__ void k_poison_flagged(const SkProblem* probs, int nprobs) {
  const float qnan = __int_as_float(0x7fc00000);
  for (int q = blockIdx.x; q < nprobs; q += gridDim.x) {
    const SkProblem& pr = probs[q];
    const int P = pr.P, K = pr.K;
    const int* range = pr.sync + 4 * P;
    const size_t N = pr.N, PN = (size_t)P * N;
    const size_t last = pr.fwd_only ? (size_t)((pr.L - 1) & 1) : (size_t)(pr.L - 1);
    for (int p = 0; p < P; ++p) {
      if (!range[p]) continue;
      float* acc = pr.acc + last * PN + (size_t)p * N;
      for (size_t j = threadIdx.x; j < N; j += blockDim.x) acc[j] = qnan;
      if (pr.fwd_only) continue;
      if (threadIdx.x == 0) pr.loss[p] = (double)qnan;
      for (int k = threadIdx.x; k < K; k += blockDim.x) pr.dot[(size_t)p * K + k] = (double)qnan;
      if (pr.need_dic) {
        float* gd = pr.gdic + (size_t)p * K * N;
        for (size_t j = threadIdx.x; j < (size_t)K * N; j += blockDim.x) gd[j] = qnan;
      }
    }
  }
}

// Per-problem sync words: done_fwd, bary_ready (0), done_bwd, msg_ready (-1),
// range (0).
__global__ void k_sync_init(int* work_err, const SkProblem* probs, int nprobs) {
  if (blockIdx.x == 0 && threadIdx.x < 2) work_err[threadIdx.x] = 0;
  for (int q = blockIdx.x; q < nprobs; q += gridDim.x) {
    const int P = probs[q].P;
    int* s = probs[q].sync;
    for (int i = threadIdx.x; i < 5 * P; i += blockDim.x) s[i] = (i >= 3 * P && i < 4 * P) ? -1 : 0;
  }
}

}  // namespace

void sk_fill_geometry(SkProblem& pr, int W, int H, bool split_bf16) {
  pr.W = W;
  pr.H = H;
  pr.Wp = (W + 15) & ~15;
  pr.Hp = (H + 15) & ~15;
  pr.N = (size_t)W * H;
  pr.vec = (W % 4) == 0;
  pr.cpr = (uint32_t)(pr.Wp / (split_bf16 ? 8 : 4));  // 16-byte operand chunks per row
  pr.cpr_magic = (uint32_t)((0x100000000ull + pr.cpr - 1) / pr.cpr);
}

size_t sk_problem_items(const SkProblem& pr) {
  const size_t PK = (size_t)pr.P * pr.K;
  if (pr.fwd_only) return (size_t)pr.L * PK;
  return (size_t)pr.L * PK * (1 + (pr.need_dic ? 2 : 1));
}

// Separable-operator applications of one problem's items: 2 per forward item,
// 2 per dictionary item (1 at step 1), 2 per weight item (none at step 1) —
// (6L-4) per atom and histogram with the dictionary recursion, (4L-2) without.
double sk_problem_applications(const SkProblem& pr) {
  const double PK = (double)pr.P * pr.K, L = pr.L;
  if (pr.fwd_only) return 2 * L * PK;
  return PK * (2 * L + (pr.need_dic ? 2 * L - 1 : 0) + 2 * (L - 1));
}

int sinkhorn_tc_launch(wdl_ctx* ctx, SkArgs& a, cudaStream_t s) {
  const size_t smem = 3 * tc::kTileBytes + 1024 + 256 + 2 * sizeof(SkProblem) + 64;
  const bool split = ctx->precision == WDL_SPLIT_BF16;
  k_sync_init<<<a.nprobs < 256 ? a.nprobs : 256, 128, 0, s>>>(a.sync, a.probs, a.nprobs);
  WDL_LAUNCH_CHECK(ctx);
  if (split)
    WDL_CUDA_TRY(ctx, cudaFuncSetAttribute(sinkhorn_tc_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  else
    WDL_CUDA_TRY(ctx, cudaFuncSetAttribute(sinkhorn_tc_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const long long streams = (a.total + 1) / 2;
  const unsigned grid = (unsigned)(streams < ctx->sm_count ? streams : ctx->sm_count);
  a.trace = nullptr;
  a.dep_wait_ns = ctx->wait_limit_s > 0 ? (unsigned long long)(ctx->wait_limit_s * 1e9) : kDepWaitNs;
  if (ctx->trace_level >= 2) {
    if (!ctx->d_trace) WDL_CUDA_TRY(ctx, cudaMalloc(&ctx->d_trace, 27 * sizeof(unsigned long long)));
    WDL_CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_trace, 0, 27 * sizeof(unsigned long long), s));
    a.trace = ctx->d_trace;
  }
  if (ctx->profiling) cudaEventRecord(ctx->ev_a, s);
  if (split) sinkhorn_tc_kernel<true><<<grid, 2 * kSt, smem, s>>>(a);
  else sinkhorn_tc_kernel<false><<<grid, 2 * kSt, smem, s>>>(a);
  WDL_LAUNCH_CHECK(ctx);
  k_poison_flagged<<<a.nprobs < 256 ? a.nprobs : 256, 256, 0, s>>>(a.probs, a.nprobs);
  WDL_LAUNCH_CHECK(ctx);
  if (ctx->profiling) {
    cudaEventRecord(ctx->ev_b, s);
    cudaEventSynchronize(ctx->ev_b);
    float ms = 0;
    cudaEventElapsedTime(&ms, ctx->ev_a, ctx->ev_b);
    ctx->conv_ms += ms;
    ctx->conv_launches += 1;
    ctx->conv_images += a.apps;
  }
  return WDL_OK;
}

// Status word of the fused kernel (sync[1]); cleared when read.
int sinkhorn_tc_status(wdl_ctx* ctx, int* sync_dev) {
  int h = 0;
  WDL_CUDA_TRY(ctx, cudaMemcpy(&h, sync_dev + 1, sizeof(int), cudaMemcpyDeviceToHost));
  if (h != 0) return set_error(ctx, h, "fused tensor-core kernel: a bounded wait timed out");
  return WDL_OK;
}

}  // namespace wdl
