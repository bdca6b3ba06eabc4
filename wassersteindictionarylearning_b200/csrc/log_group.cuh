// The stabilised log-sum-exp of one group of four neighbouring outputs of a
// staged row (the separable log-domain operator's inner computation), shared
// by the CUDA-core operator's axis pass (conv_simt.cu) and the persistent
// log-domain weight fits (fit_log.cu).  out = log |sum_k s_k exp(-(c-k)^2/gamma
// + row[k])| for c = c0..c0+3 (cpp/kernels.h:1082-1091, signed :1123-1136),
// one pass with a running maximum, taps outwards from the centres.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace wdl {
namespace lse {

template <typename T>
struct LogOps;
template <>
struct LogOps<float> {
  static constexpr float kScale = 1.4426950408889634f;   // log2 e: natural -> base 2
  static constexpr float kUnscale = 0.6931471805599453f;  // ln 2
  static constexpr float kTail = 40.f;                   // bits
  static constexpr float kFloor = -3.402823466e38f;      // lowest start of a maximum
  static constexpr float kNone = -__builtin_huge_valf();  // a tap outside the row
  // the hardware base-2 exponential; arguments are <= 0 here (up to rounding)
  // and results below 2^-126 are far under the sum's rounding, so flushing them
  // is exact
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
  static constexpr double kNone = -__builtin_huge_val();
  __device__ static double ex(double x) { return exp(x); }
  __device__ static double lg(double x) { return log(x); }
};

// Rows are staged with kHalo taps of kNone on each side, so the loads of a
// group need no range test while d <= c0 + kHalo on the left and
// c0 + 3 + d < C + kHalo on the right.
constexpr int kHalo = 8;

// +1 for sign byte 1, -1 for sign byte 0 (sign bytes are 0 or 1 throughout):
// one integer multiply-add on the bit pattern of -1.
template <typename T>
__device__ __forceinline__ T sign_of(uint8_t b);
template <>
__device__ __forceinline__ float sign_of<float>(uint8_t b) {
  return __uint_as_float(0xBF800000u + (uint32_t)b * 0x80000000u);
}
template <>
__device__ __forceinline__ double sign_of<double>(uint8_t b) {
  return __longlong_as_double((long long)(0xBFF0000000000000ull + (unsigned long long)b * 0x8000000000000000ull));
}

// The state of one group of four outputs: running maxima m[j] and sums s[j],
// and the taps of the current step in two 4-entry rings indexed by row
// position mod 4 (left taps in lq, right taps in rq; their signs as +-1 in lsg
// and rsg).  At distance d output j reads lq[(j - d) & 3] and rq[(j + d) & 3].
template <typename T>
struct LogGroup {
  T m[4], s[4];
  T lq[4], rq[4];
  T lsg[4], rsg[4];
  T mmin;   // min over the group's outputs of m
  T mtail;  // mmin - kTail
};

template <typename T>
__device__ __forceinline__ T vmax(T a, T b) { return fmax(a, b); }
template <>
__device__ __forceinline__ float vmax<float>(float a, float b) { return fmaxf(a, b); }
template <typename T>
__device__ __forceinline__ T vmin(T a, T b) { return fmin(a, b); }
template <>
__device__ __forceinline__ float vmin<float>(float a, float b) { return fminf(a, b); }

template <typename T, bool FULL>
__device__ __forceinline__ void log_group_mmin(LogGroup<T>& g, int nv) {
  T mn = g.m[0];
#pragma unroll
  for (int j = 1; j < 4; ++j)
    if (FULL || j < nv) mn = vmin(mn, g.m[j]);
  g.mmin = mn;
  g.mtail = mn - LogOps<T>::kTail;
}

// The terms of one step at distance d (d & 3 == DM) whose two new taps are in
// the rings: l = lk[d], bound = l + X.
template <typename T, bool SIGNED, bool FULL, int DM>
__device__ __forceinline__ void log_group_terms(LogGroup<T>& g, T l, T bound, int nv) {
  using Op = LogOps<T>;
  T a[4], b[4], t[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const T lm = l - g.m[j];
    a[j] = g.lq[(j - DM) & 3] + lm;
    b[j] = g.rq[(j + DM) & 3] + lm;
  }
  // A new maximum is possible only while the bound exceeds some output's
  // maximum; then shift the sums of the outputs that found one (t = 0 leaves
  // an output unchanged).
  if (bound > g.mmin) {
    bool up = false;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      t[j] = vmax(a[j], b[j]);
      up |= t[j] > T(0);
    }
    if (up) {
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const T tj = vmax(t[j], T(0));
        g.s[j] *= Op::ex(-tj);
        g.m[j] += tj;
        a[j] -= tj;
        b[j] -= tj;
      }
      log_group_mmin<T, FULL>(g, nv);
    }
  }
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    if (SIGNED) {
      g.s[j] += g.lsg[(j - DM) & 3] * Op::ex(a[j]);
      g.s[j] += g.rsg[(j + DM) & 3] * Op::ex(b[j]);
    } else {
      g.s[j] += Op::ex(a[j]);
      g.s[j] += Op::ex(b[j]);
    }
  }
}

// Step d = d0 + K (d & 3 == DM) of a block of four inside the halo: the taps
// come from lp[-K] and rp[K] (lp = row + c0 - d0, rp = row + c0 + 3 + d0) and
// the weight from lkp[K] (lkp = lk + d0), immediate offsets from one base per
// block.  False once every output of the group has its sum.
template <typename T, bool SIGNED, bool FULL, int DM, int K>
__device__ __forceinline__ bool log_group_step(LogGroup<T>& g, const T* lkp, const T* lp, const T* rp,
                                               const uint8_t* lsp, const uint8_t* rsp, T X, int nv) {
  const T l = lkp[K];
  const T bound = l + X;  // no tap at distance >= d has a larger exponent
  if (bound < g.mtail) return false;
  constexpr int il = (4 - DM) & 3, ir = (3 + DM) & 3;  // ring slots of positions c0 - d, c0 + 3 + d
  g.lq[il] = lp[-K];
  g.rq[ir] = rp[K];
  if (SIGNED) {
    g.lsg[il] = sign_of<T>(lsp[-K]);
    g.rsg[ir] = sign_of<T>(rsp[K]);
  }
  log_group_terms<T, SIGNED, FULL, DM>(g, l, bound, nv);
  return true;
}

// Step d (d & 3 == DM) whose taps may lie beyond the halo.
template <typename T, bool SIGNED, bool FULL, int DM>
__device__ __forceinline__ bool log_group_step_guarded(LogGroup<T>& g, const T* __restrict__ row,
                                                       const uint8_t* __restrict__ sgn,
                                                       const T* __restrict__ lk, T X, int c0, int C, int d,
                                                       int nv) {
  using Op = LogOps<T>;
  const T l = lk[d];
  const T bound = l + X;
  if (bound < g.mtail) return false;
  const int pl = c0 - d, pr = c0 + 3 + d;
  constexpr int il = (4 - DM) & 3, ir = (3 + DM) & 3;
  g.lq[il] = pl >= 0 ? row[pl] : Op::kNone;
  g.rq[ir] = pr < C ? row[pr] : Op::kNone;
  if (SIGNED) {
    g.lsg[il] = pl >= 0 ? sign_of<T>(sgn[pl]) : T(1);
    g.rsg[ir] = pr < C ? sign_of<T>(sgn[pr]) : T(1);
  }
  log_group_terms<T, SIGNED, FULL, DM>(g, l, bound, nv);
  return true;
}

// Outputs c0..c0+3 of one staged row (row[-kHalo..C+kHalo) readable; those
// below C are valid; FULL: all four are): v[j] and, when SIGNED, pos[j]
// (sum >= 0).  Returns the exponentials evaluated per output.
template <typename T, bool SIGNED, bool FULL>
__device__ __forceinline__ int log_group(const T* __restrict__ row, const uint8_t* __restrict__ sgn,
                                         const T* __restrict__ lk, T X, int c0, int C, T* v, bool* pos) {
  using Op = LogOps<T>;
  LogGroup<T> g;
  const int nv = FULL ? 4 : min(4, C - c0);
  // row positions c0-1 .. c0+4 (inside the halo: kNone beyond the row)
  T x[6], sx[6];
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    x[i] = row[c0 - 1 + i];
    sx[i] = SIGNED ? sign_of<T>(sgn[c0 - 1 + i]) : T(1);
  }
  // distances 0 and 1: m = max(centre, neighbours + lk[1], floor)
  const T l1 = C > 1 ? lk[1] : Op::kNone;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const T cx = x[j + 1], lx = x[j], rx = x[j + 2];
    const T m = vmax(vmax(cx, Op::kFloor), vmax(lx, rx) + l1);
    const T lm = l1 - m;
    T s = SIGNED ? sx[j + 1] * Op::ex(cx - m) : Op::ex(cx - m);
    if (SIGNED) {
      s += sx[j] * Op::ex(lx + lm);
      s += sx[j + 2] * Op::ex(rx + lm);
    } else {
      s += Op::ex(lx + lm);
      s += Op::ex(rx + lm);
    }
    g.m[j] = m;
    g.s[j] = s;
  }
  // rings for distance 1 (left taps at c0-1..c0+2, right taps at c0+1..c0+4)
  g.lq[0] = x[1]; g.lq[1] = x[2]; g.lq[2] = x[3]; g.lq[3] = x[0];
  g.rq[0] = x[5]; g.rq[1] = x[2]; g.rq[2] = x[3]; g.rq[3] = x[4];
  if (SIGNED) {
    g.lsg[0] = sx[1]; g.lsg[1] = sx[2]; g.lsg[2] = sx[3]; g.lsg[3] = sx[0];
    g.rsg[0] = sx[5]; g.rsg[1] = sx[2]; g.rsg[2] = sx[3]; g.rsg[3] = sx[4];
  }
  log_group_mmin<T, FULL>(g, nv);
  // beyond dend every tap of every valid output lies outside the row; up to
  // dsafe both new taps of a step lie inside the halo
  const int dend = max(min(c0 + 3, C - 1), C - 1 - c0);
  const int dsafe = min(dend, min(c0 + kHalo, C + kHalo - 4 - c0));
  int d = 2;
  bool done = false;
  // blocks of four steps inside the halo (d = 2 mod 4 at each block's start)
  while (d + 3 <= dsafe) {
    const T* lkp = lk + d;
    const T* lp = row + (c0 - d);
    const T* rp = row + (c0 + 3 + d);
    const uint8_t* lsp = SIGNED ? sgn + (c0 - d) : nullptr;
    const uint8_t* rsp = SIGNED ? sgn + (c0 + 3 + d) : nullptr;
    if (!log_group_step<T, SIGNED, FULL, 2, 0>(g, lkp, lp, rp, lsp, rsp, X, nv)) { done = true; break; }
    if (!log_group_step<T, SIGNED, FULL, 3, 1>(g, lkp, lp, rp, lsp, rsp, X, nv)) { done = true; d += 1; break; }
    if (!log_group_step<T, SIGNED, FULL, 0, 2>(g, lkp, lp, rp, lsp, rsp, X, nv)) { done = true; d += 2; break; }
    if (!log_group_step<T, SIGNED, FULL, 1, 3>(g, lkp, lp, rp, lsp, rsp, X, nv)) { done = true; d += 3; break; }
    d += 4;
  }
  // the remaining steps, with range tests
  for (; !done && d <= dend; ++d) {
    bool go;
    switch (d & 3) {
      case 0: go = log_group_step_guarded<T, SIGNED, FULL, 0>(g, row, sgn, lk, X, c0, C, d, nv); break;
      case 1: go = log_group_step_guarded<T, SIGNED, FULL, 1>(g, row, sgn, lk, X, c0, C, d, nv); break;
      case 2: go = log_group_step_guarded<T, SIGNED, FULL, 2>(g, row, sgn, lk, X, c0, C, d, nv); break;
      default: go = log_group_step_guarded<T, SIGNED, FULL, 3>(g, row, sgn, lk, X, c0, C, d, nv); break;
    }
    if (!go) break;
  }
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    if (SIGNED) {
      pos[j] = g.s[j] >= T(0);
      v[j] = (Op::lg(fabs(g.s[j])) + g.m[j]) * Op::kUnscale;
    } else {
      pos[j] = true;
      v[j] = (Op::lg(g.s[j]) + g.m[j]) * Op::kUnscale;
    }
  }
  return 3 + 2 * (d - 2);
}


// SMEM row strides: values C + 2 kHalo + 1 (odd), sign bytes C + 2 kHalo + 4.
__host__ __device__ constexpr int log_cp(int C) { return C + 2 * kHalo + 1; }
__host__ __device__ constexpr int log_sp(int C) { return C + 2 * kHalo + 4; }

}  // namespace lse
}  // namespace wdl
