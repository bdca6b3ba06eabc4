/* Test infrastructure only — CPU oracle (FP64) for the Sinkhorn-barycenter hot
 * path.  See wdl_oracle.h for the contract.  Every routine restates the
 * reference algorithm at the file:line cited beside it, keeping its order of
 * summation so that results agree with the reference to rounding.
 */
#include "wdl_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static double* xalloc(size_t n) {
  double* p = (double*)calloc(n ? n : 1, sizeof(double));
  if (!p) abort();
  return p;
}

static inline double safe_log(double x) { /* cpp/loss.h:3-5 */
  return log(x > ORC_EPSILON ? x : ORC_EPSILON);
}

void orc_kernel1d(double gamma, int n, double* out) { /* cpp/kernels.h:637-640 */
  for (int i = 0; i < n; ++i) {
    double v = exp(-(i * i) / gamma);
    out[i] = v > ORC_EPSILON ? v : ORC_EPSILON;
  }
}

/* One axis of the separable operator: in is [R][C] (C contiguous), out is
 * [C][R]: the contracted axis moves to the front.  Applying it once per axis
 * returns the image to its original layout; each output sums k = 0..C-1 in
 * order, as the reference's passes do (cpp/kernels.h:677-697). */
static void axis_pass(const double* in, double* out, int R, int C, const double* k1d) {
  for (int r = 0; r < R; ++r) {
    const double* row = in + (size_t)r * C;
    for (int c = 0; c < C; ++c) {
      double acc = 0;
      for (int k = 0; k < C; ++k) acc += k1d[abs(c - k)] * row[k];
      out[(size_t)c * R + r] = acc;
    }
  }
}

void orc_convolve(int W, int H, int D, double gamma, const double* u, double* out, int nv) {
  const size_t N = (size_t)W * H * D;
  int M = W > H ? W : H;
  if (D > M) M = D;
  double* k1d = xalloc(M);
  orc_kernel1d(gamma, M, k1d);
  double* t1 = xalloc(N);
  double* t2 = xalloc(N);
  for (int v = 0; v < nv; ++v) {
    const double* src = u + v * N;
    double* dst = out + v * N;
    if (D == 1) { /* cpp/kernels.h:669-699 */
      axis_pass(src, t1, H, W, k1d);
      axis_pass(t1, dst, W, H, k1d);
    } else { /* cpp/kernels.h:762-807 */
      axis_pass(src, t1, D * H, W, k1d);
      axis_pass(t1, t2, W * D, H, k1d);
      axis_pass(t2, dst, H * W, D, k1d);
    }
  }
  free(k1d);
  free(t1);
  free(t2);
}

/* Log-domain axis pass (cpp/kernels.h:1079-1092): max pass then exp-sum pass.
 * With signs != NULL the terms carry the input signs (bit=1 means >= 0) and
 * the output sign is written to out_signs (cpp/kernels.h:1123-1136). */
static inline int get_sign(const unsigned char* t, size_t i) { return ((t[i / 8] >> (i % 8)) & 1) ? 1 : -1; }
static inline void set_sign(unsigned char* t, size_t i, double v) {
  if (v >= 0) t[i / 8] |= (unsigned char)(1u << (i % 8));
  else t[i / 8] &= (unsigned char)~(1u << (i % 8));
}

static void log_axis_pass(const double* in, double* out, int R, int C, double gamma,
                          const unsigned char* in_signs, size_t in_sign_base,
                          unsigned char* out_signs, size_t out_sign_base) {
  for (int r = 0; r < R; ++r) {
    const double* row = in + (size_t)r * C;
    for (int c = 0; c < C; ++c) {
      double vmax = -1e99;
      for (int k = 0; k < C; ++k) {
        double t = -((c - k) * (c - k)) / gamma + row[k];
        vmax = vmax > t ? vmax : t;
      }
      double conv = 0;
      for (int k = 0; k < C; ++k) {
        double e = exp(-((c - k) * (c - k)) / gamma + row[k] - vmax);
        if (in_signs) e = get_sign(in_signs, in_sign_base + (size_t)r * C + k) * e;
        conv += e;
      }
      size_t o = (size_t)c * R + r;
      if (out_signs) {
        set_sign(out_signs, out_sign_base + o, conv);
        out[o] = log(fabs(conv)) + vmax;
      } else {
        out[o] = log(conv) + vmax;
      }
    }
  }
}

void orc_log_convolve(int W, int H, double gamma, const double* log_u, double* out, int nv) {
  const size_t N = (size_t)W * H;
  double* t = xalloc(N);
  for (int v = 0; v < nv; ++v) {
    log_axis_pass(log_u + v * N, t, H, W, gamma, NULL, 0, NULL, 0);
    log_axis_pass(t, out + v * N, W, H, gamma, NULL, 0, NULL, 0);
  }
  free(t);
}

void orc_log_convolve_signed(int W, int H, double gamma, const double* log_u,
                             unsigned char* signs, double* out, int nv) {
  const size_t N = (size_t)W * H;
  double* t = xalloc(N);
  unsigned char* ts = (unsigned char*)calloc((N + 7) / 8, 1);
  for (int v = 0; v < nv; ++v) {
    /* x-pass: image v's input signs live at v*N; the transposed temp keeps its own. */
    log_axis_pass(log_u + v * N, t, H, W, gamma, signs, v * N, ts, 0);
    log_axis_pass(t, out + v * N, W, H, gamma, ts, 0, signs, v * N);
  }
  free(t);
  free(ts);
}

/* Wasserstein loss helper: the entropic OT scalings of cpp/loss.h:102-118. */
static void w_scalings(int W, int H, int D, double gamma, const double* v1, const double* v2,
                       int n_iter, double* a, double* b, double* conv) {
  const size_t N = (size_t)W * H * D;
  for (size_t j = 0; j < N; ++j) a[j] = b[j] = 1.0;
  for (int it = 0; it < n_iter; ++it) {
    orc_convolve(W, H, D, gamma, b, conv, 1);
    for (size_t j = 0; j < N; ++j) a[j] = v1[j] / conv[j];
    orc_convolve(W, H, D, gamma, a, conv, 1);
    for (size_t j = 0; j < N; ++j) b[j] = v2[j] / conv[j];
  }
}

double orc_loss(int loss_type, int W, int H, int D, double gamma, const double* v1,
                const double* v2, double* grad) {
  const size_t N = (size_t)W * H * D;
  double r = 0;
  switch (loss_type) {
    case 1: /* TV, cpp/loss.h:43-66 */
      for (size_t i = 0; i < N; ++i) {
        double d = v1[i] - v2[i];
        r += fabs(d);
        if (grad) grad[i] = d > 0 ? 0.5 : -0.5;
      }
      return 0.5 * r;
    case 2: /* quadratic, cpp/loss.h:19-41 */
      for (size_t i = 0; i < N; ++i) {
        double d = v1[i] - v2[i];
        r += d * d;
        if (grad) grad[i] = 2. * (v1[i] - v2[i]);
      }
      return r;
    case 4: /* KL, cpp/loss.h:68-90 */
      for (size_t i = 0; i < N; ++i) {
        r += v1[i] * safe_log(v1[i] / v2[i]) - v1[i] + v2[i];
        if (grad) grad[i] = safe_log(v1[i] / v2[i]);
      }
      return r;
    case 3: { /* Wasserstein, cpp/loss.h:92-154, 50 inner iterations */
      double* a = xalloc(N);
      double* b = xalloc(N);
      double* c = xalloc(N);
      w_scalings(W, H, D, gamma, v1, v2, 50, a, b, c);
      orc_convolve(W, H, D, gamma, b, c, 1);
      for (size_t j = 0; j < N; ++j) r += safe_log(a[j]) * v1[j] + safe_log(b[j]) * v2[j] - a[j] * c[j];
      if (grad)
        for (size_t j = 0; j < N; ++j) grad[j] = gamma * safe_log(a[j]);
      free(a);
      free(b);
      free(c);
      return gamma * r;
    }
    default:
      return NAN;
  }
}

static void normalized_copy(const double* atoms, const double* lambdas, int K, size_t N,
                            double* p, double* lam) {
  double s = 0; /* Problem::normalize_values, cpp/inverseWasserstein.h:53-74 */
  for (int i = 0; i < K; ++i) s += lambdas[i];
  for (int i = 0; i < K; ++i) lam[i] = lambdas[i] / s;
  for (int i = 0; i < K; ++i) {
    double s2 = 0;
    for (size_t j = 0; j < N; ++j) s2 += atoms[i * N + j];
    for (size_t j = 0; j < N; ++j) p[i * N + j] = atoms[i * N + j] / s2;
  }
}

static void gradient_both_impl(int W, int H, int D, double gamma, int K, int L, int loss_type,
                               const double* atoms, const double* lambdas, const double* obs,
                               const double* b_init, double* resultLa, double* resultDic,
                               double* bary, double* b_last, double* la_abs) {
  const size_t N = (size_t)W * H * D, KN = (size_t)K * N;
  double* p = xalloc(KN);
  double* lam = xalloc(K);
  normalized_copy(atoms, lambdas, K, N, p, lam);
  double* b = xalloc((L + 1) * KN);
  double* conv_b = xalloc(L * KN);
  double* phi = xalloc((L + 1) * KN);
  double* a = xalloc(KN);
  double* g = xalloc(N);
  for (size_t i = 0; i < KN; ++i) b[i] = b_init ? b_init[i] : 1.0;

  /* Forward Bregman projections with tape, cpp/inverseWasserstein.h:565-593. */
  for (int it = 1; it <= L; ++it) {
    double* cb = conv_b + (size_t)(it - 1) * KN;
    double* ph = phi + (size_t)it * KN;
    orc_convolve(W, H, D, gamma, b + (size_t)(it - 1) * KN, cb, K);
    for (size_t i = 0; i < KN; ++i) a[i] = p[i] / cb[i];
    orc_convolve(W, H, D, gamma, a, ph, K);
    for (size_t j = 0; j < N; ++j) bary[j] = 0;
    for (int k = 0; k < K; ++k)
      for (size_t j = 0; j < N; ++j) bary[j] += safe_log(ph[k * N + j]) * lam[k];
    for (size_t j = 0; j < N; ++j) bary[j] = exp(bary[j]);
    for (int k = 0; k < K; ++k)
      for (size_t j = 0; j < N; ++j) b[(size_t)it * KN + k * N + j] = bary[j] / ph[k * N + j];
  }
  if (b_last) memcpy(b_last, b + (size_t)L * KN, KN * sizeof(double));

  orc_loss(loss_type, W, H, D, gamma, bary, obs, g); /* :597 */

  /* Dictionary gradient, :602-629. */
  double* n = xalloc(N);
  double* v = xalloc(KN);
  double* tmp = xalloc(KN);
  double* c = xalloc(KN);
  double* sumv = xalloc(N);
  memset(resultDic, 0, KN * sizeof(double));
  memcpy(n, g, N * sizeof(double));
  for (int s = L; s >= 1; --s) {
    const double* bs = b + (size_t)s * KN;
    const double* cb = conv_b + (size_t)(s - 1) * KN;
    for (size_t j = 0; j < N; ++j) sumv[j] = 0;
    for (int k = 0; k < K; ++k)
      for (size_t j = 0; j < N; ++j)
        tmp[k * N + j] = (lam[k] * n[j] - v[k * N + j]) * bs[k * N + j];
    orc_convolve(W, H, D, gamma, tmp, c, K);
    for (size_t i = 0; i < KN; ++i) {
      resultDic[i] += c[i] / cb[i];
      tmp[i] = -p[i] * c[i] / (cb[i] * cb[i]);
    }
    if (s == 1) break;
    orc_convolve(W, H, D, gamma, tmp, v, K);
    const double* ph = phi + (size_t)(s - 1) * KN;
    for (int k = 0; k < K; ++k)
      for (size_t j = 0; j < N; ++j) {
        v[k * N + j] /= ph[k * N + j];
        sumv[j] += v[k * N + j];
      }
    memcpy(n, sumv, N * sizeof(double));
  }

  /* Weight gradient, :635-673. */
  for (size_t j = 0; j < N; ++j) g[j] *= bary[j];
  double* r = xalloc(KN);
  double* u = xalloc(KN);
  double* convu = xalloc(KN);
  for (int k = 0; k < K; ++k) resultLa[k] = 0;
  if (la_abs)
    for (int k = 0; k < K; ++k) la_abs[k] = 0;
  for (int s = L; s >= 1; --s) {
    const double* ph = phi + (size_t)s * KN;
    for (int k = 0; k < K; ++k) {
      double dotp = 0;
      for (size_t j = 0; j < N; ++j) {
        if (la_abs) la_abs[k] += fabs(log(ph[k * N + j]) * g[j]);
        dotp += log(ph[k * N + j]) * g[j];
        u[k * N + j] = (lam[k] * g[j] - r[k * N + j]) / ph[k * N + j];
      }
      resultLa[k] += dotp;
    }
    if (s != 1) {
      const double* cb = conv_b + (size_t)(s - 1) * KN;
      const double* bp = b + (size_t)(s - 1) * KN;
      orc_convolve(W, H, D, gamma, u, convu, K);
      for (size_t i = 0; i < KN; ++i) convu[i] *= -p[i] / (cb[i] * cb[i]);
      orc_convolve(W, H, D, gamma, convu, r, K);
      for (size_t i = 0; i < KN; ++i) r[i] *= bp[i];
      for (size_t j = 0; j < N; ++j) g[j] = 0;
      for (int k = 0; k < K; ++k)
        for (size_t j = 0; j < N; ++j) g[j] += r[k * N + j];
    }
  }
  free(p); free(lam); free(b); free(conv_b); free(phi); free(a); free(g);
  free(n); free(v); free(tmp); free(c); free(sumv); free(r); free(u); free(convu);
}

static inline double abs_log(double val, unsigned char* s, size_t i) { /* cpp/signArray.h:24-29 */
  set_sign(s, i, val);
  return log(fabs(val));
}
static inline double abs_exp(double lv, const unsigned char* s, size_t i) { /* :31-35 */
  return get_sign(s, i) * exp(lv);
}

static void gradient_both_log_impl(int W, int H, double gamma, int K, int L, int loss_type,
                                   const double* atoms, const double* lambdas, const double* obs,
                                   double* resultLa, double* resultDic, double* bary,
                                   double* la_abs) {
  const size_t N = (size_t)W * H, KN = (size_t)K * N;
  double* p = xalloc(KN);
  double* lam = xalloc(K);
  normalized_copy(atoms, lambdas, K, N, p, lam);
  double* b = xalloc((L + 1) * KN); /* b[0] = 0 (log of ones), :687 */
  double* conv_b = xalloc(L * KN);
  double* phi = xalloc((L + 1) * KN);
  double* a = xalloc(KN);
  double* g = xalloc(N);
  /* Forward, :700-720. */
  for (int it = 1; it <= L; ++it) {
    double* cb = conv_b + (size_t)(it - 1) * KN;
    double* ph = phi + (size_t)it * KN;
    orc_log_convolve(W, H, gamma, b + (size_t)(it - 1) * KN, cb, K);
    for (size_t i = 0; i < KN; ++i) a[i] = log(p[i]) - cb[i];
    orc_log_convolve(W, H, gamma, a, ph, K);
    for (size_t j = 0; j < N; ++j) bary[j] = 0;
    for (int k = 0; k < K; ++k)
      for (size_t j = 0; j < N; ++j) bary[j] += ph[k * N + j] * lam[k];
    for (int k = 0; k < K; ++k)
      for (size_t j = 0; j < N; ++j) b[(size_t)it * KN + k * N + j] = bary[j] - ph[k * N + j];
  }
  for (size_t j = 0; j < N; ++j) bary[j] = exp(bary[j]);
  orc_loss(loss_type, W, H, 1, gamma, bary, obs, g);

  /* Dictionary gradient with one shared sign array, :730-765.  v holds -v. */
  double* n = xalloc(N);
  double* v = xalloc(KN);
  double* tmp = xalloc(KN);
  double* c = xalloc(KN);
  double* sumv = xalloc(N);
  unsigned char* sg = (unsigned char*)calloc((KN + 7) / 8, 1);
  memset(resultDic, 0, KN * sizeof(double));
  memcpy(n, g, N * sizeof(double));
  for (int s = L; s >= 1; --s) {
    const double* cb = conv_b + (size_t)(s - 1) * KN;
    for (size_t j = 0; j < N; ++j) sumv[j] = 0;
    for (int k = 0; k < K; ++k)
      for (size_t j = 0; j < N; ++j) {
        size_t i = k * N + j;
        tmp[i] = abs_log(lam[k] * n[j] + v[i], sg, i) + b[(size_t)s * KN + i];
      }
    orc_log_convolve_signed(W, H, gamma, tmp, sg, c, K);
    for (size_t i = 0; i < KN; ++i) {
      resultDic[i] += abs_exp(c[i] - cb[i], sg, i);
      tmp[i] = log(p[i]) + c[i] - 2.0 * cb[i];
    }
    if (s == 1) break;
    orc_log_convolve_signed(W, H, gamma, tmp, sg, v, K);
    const double* ph = phi + (size_t)(s - 1) * KN;
    for (int k = 0; k < K; ++k)
      for (size_t j = 0; j < N; ++j) {
        size_t i = k * N + j;
        v[i] = abs_exp(v[i] - ph[i], sg, i);
        sumv[j] -= v[i];
      }
    memcpy(n, sumv, N * sizeof(double));
  }

  /* Weight gradient, :770-812.  r holds -r. */
  for (size_t j = 0; j < N; ++j) g[j] *= bary[j];
  double* r = xalloc(KN);
  double* u = xalloc(KN);
  double* convu = xalloc(KN);
  for (int k = 0; k < K; ++k) resultLa[k] = 0;
  if (la_abs)
    for (int k = 0; k < K; ++k) la_abs[k] = 0;
  for (int s = L; s >= 1; --s) {
    const double* ph = phi + (size_t)s * KN;
    for (int k = 0; k < K; ++k) {
      double dotp = 0;
      for (size_t j = 0; j < N; ++j) {
        size_t i = k * N + j;
        if (la_abs) la_abs[k] += fabs(ph[i] * g[j]);
        dotp += ph[i] * g[j];
        u[i] = abs_log(lam[k] * g[j] + r[i], sg, i) - ph[i];
      }
      resultLa[k] += dotp;
    }
    if (s != 1) {
      const double* cb = conv_b + (size_t)(s - 1) * KN;
      const double* bp = b + (size_t)(s - 1) * KN;
      orc_log_convolve_signed(W, H, gamma, u, sg, convu, K);
      for (size_t i = 0; i < KN; ++i) convu[i] += log(p[i]) - 2.0 * cb[i];
      orc_log_convolve_signed(W, H, gamma, convu, sg, r, K);
      for (size_t i = 0; i < KN; ++i) r[i] = abs_exp(r[i] + bp[i], sg, i);
      for (size_t j = 0; j < N; ++j) g[j] = 0;
      for (int k = 0; k < K; ++k)
        for (size_t j = 0; j < N; ++j) g[j] -= r[k * N + j];
    }
  }
  free(sg);
  free(p); free(lam); free(b); free(conv_b); free(phi); free(a); free(g);
  free(n); free(v); free(tmp); free(c); free(sumv); free(r); free(u); free(convu);
}

void orc_gradient_both(int W, int H, int D, double gamma, int K, int L, int loss_type,
                       const double* atoms, const double* lambdas, const double* obs,
                       const double* b_init, double* resultLa, double* resultDic,
                       double* bary, double* b_last) {
  gradient_both_impl(W, H, D, gamma, K, L, loss_type, atoms, lambdas, obs, b_init, resultLa,
                     resultDic, bary, b_last, NULL);
}

void orc_gradient_both_log(int W, int H, double gamma, int K, int L, int loss_type,
                           const double* atoms, const double* lambdas, const double* obs,
                           double* resultLa, double* resultDic, double* bary) {
  gradient_both_log_impl(W, H, gamma, K, L, loss_type, atoms, lambdas, obs, resultLa, resultDic,
                         bary, NULL);
}

void orc_gradient_both_scale(int W, int H, int D, double gamma, int K, int L, int loss_type,
                             int log_domain, const double* atoms, const double* lambdas,
                             const double* obs, double* la_abs) {
  const size_t N = (size_t)W * H * D;
  double* la = xalloc(K);
  double* dic = xalloc((size_t)K * N);
  double* bary = xalloc(N);
  if (log_domain)
    gradient_both_log_impl(W, H, gamma, K, L, loss_type, atoms, lambdas, obs, la, dic, bary, la_abs);
  else
    gradient_both_impl(W, H, D, gamma, K, L, loss_type, atoms, lambdas, obs, NULL, la, dic, bary,
                       NULL, la_abs);
  free(la);
  free(dic);
  free(bary);
}

void orc_barycenter(int W, int H, int D, double gamma, int K, int L, const double* atoms,
                    const double* lambdas, double* bary) {
  const size_t N = (size_t)W * H * D, KN = (size_t)K * N;
  double* p = xalloc(KN);
  double* lam = xalloc(K);
  normalized_copy(atoms, lambdas, K, N, p, lam);
  double* b = xalloc(KN);
  double* a = xalloc(KN);
  double* conv = xalloc(KN);
  for (size_t i = 0; i < KN; ++i) b[i] = 1.0; /* :115-119 */
  for (int it = 0; it < L; ++it) {            /* :130-152 */
    orc_convolve(W, H, D, gamma, b, conv, K);
    for (size_t i = 0; i < KN; ++i) a[i] = p[i] / conv[i];
    orc_convolve(W, H, D, gamma, a, conv, K);
    for (size_t j = 0; j < N; ++j) bary[j] = 0; /* geomMean, :296-312 */
    for (int k = 0; k < K; ++k)
      for (size_t j = 0; j < N; ++j) bary[j] += safe_log(conv[k * N + j]) * lam[k];
    for (size_t j = 0; j < N; ++j) bary[j] = exp(bary[j]);
    for (int k = 0; k < K; ++k)
      for (size_t j = 0; j < N; ++j) b[k * N + j] = bary[j] / conv[k * N + j];
  }
  free(p); free(lam); free(b); free(a); free(conv);
}

void orc_barycenter_log(int W, int H, double gamma, int K, int L, const double* atoms,
                        const double* lambdas, double* bary) {
  const size_t N = (size_t)W * H, KN = (size_t)K * N;
  double* p = xalloc(KN);
  double* lam = xalloc(K);
  normalized_copy(atoms, lambdas, K, N, p, lam);
  double* b = xalloc(KN); /* zeros = log of ones, :162 */
  double* a = xalloc(KN);
  double* conv = xalloc(KN);
  for (int it = 0; it < L; ++it) { /* :167-196 */
    orc_log_convolve(W, H, gamma, b, conv, K);
    for (size_t i = 0; i < KN; ++i) a[i] = log(p[i]) - conv[i];
    orc_log_convolve(W, H, gamma, a, conv, K);
    for (size_t j = 0; j < N; ++j) bary[j] = 0;
    for (int k = 0; k < K; ++k)
      for (size_t j = 0; j < N; ++j) bary[j] += conv[k * N + j] * lam[k];
    for (int k = 0; k < K; ++k)
      for (size_t j = 0; j < N; ++j) b[k * N + j] = bary[j] - conv[k * N + j];
  }
  for (size_t j = 0; j < N; ++j) bary[j] = exp(bary[j]);
  free(p); free(lam); free(b); free(a); free(conv);
}

double orc_evaluate_both(int W, int H, int D, double gamma, int P, int K, int L, int loss_type,
                         int log_domain, double scale_dic, const double* x, double* g,
                         const double* obs, const double* b_storage, double* b_last,
                         double* bary_out, int nthreads) {
  const size_t N = (size_t)W * H * D, KN = (size_t)K * N, PK = (size_t)P * K;
  const size_t n = PK + KN;
  double* v2 = xalloc(n);
  /* Back to the original domain and normalise, :997-1031. */
  for (size_t i = 0; i < PK; ++i) v2[i] = exp(x[i] / scale_dic);
  for (size_t i = 0; i < KN; ++i) v2[PK + i] = exp(x[PK + i]);
  for (int i = 0; i < P; ++i) {
    double s = 0;
    for (int j = 0; j < K; ++j) s += v2[i * K + j];
    for (int j = 0; j < K; ++j) v2[i * K + j] /= s;
  }
  for (int i = 0; i < K; ++i) {
    double s = 0;
    for (size_t j = 0; j < N; ++j) s += v2[PK + i * N + j];
    for (size_t j = 0; j < N; ++j) v2[PK + i * N + j] /= s;
  }
  memset(g, 0, n * sizeof(double));
  double* gdic = xalloc((size_t)P * KN);
  double* losses = xalloc(P);
  const double* atoms = v2 + PK;
#ifdef _OPENMP
  if (nthreads < 1) nthreads = 1;
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
#endif
  for (int id = 0; id < P; ++id) { /* :1052-1113 */
    double* bary = xalloc(N);
    double* gd = gdic + (size_t)id * KN;
    if (log_domain)
      orc_gradient_both_log(W, H, gamma, K, L, loss_type, atoms, v2 + (size_t)id * K,
                            obs + (size_t)id * N, g + (size_t)id * K, gd, bary);
    else
      orc_gradient_both(W, H, D, gamma, K, L, loss_type, atoms, v2 + (size_t)id * K,
                        obs + (size_t)id * N, b_storage ? b_storage + (size_t)id * KN : NULL,
                        g + (size_t)id * K, gd, bary, b_last ? b_last + (size_t)id * KN : NULL);
    losses[id] = orc_loss(loss_type, W, H, D, gamma, bary, obs + (size_t)id * N, NULL);
    double dotP = 0;
    for (int i = 0; i < K; ++i) dotP += v2[id * K + i] * g[id * K + i];
    for (int i = 0; i < K; ++i) g[id * K + i] -= dotP;
    for (int i = 0; i < K; ++i) {
      double d2 = 0;
      for (size_t j = 0; j < N; ++j) d2 += atoms[i * N + j] * gd[i * N + j];
      for (size_t j = 0; j < N; ++j) gd[i * N + j] -= d2;
    }
    if (bary_out) memcpy(bary_out + (size_t)id * N, bary, N * sizeof(double));
    free(bary);
  }
  double lossVal = 0;
  for (int id = 0; id < P; ++id) {
    lossVal += losses[id];
    for (size_t i = 0; i < KN; ++i) g[PK + i] += gdic[(size_t)id * KN + i];
  }
  for (size_t i = 0; i < n; ++i) g[i] *= v2[i]; /* chain rule, :1125-1128 */
  for (size_t i = 0; i < PK; ++i) g[i] /= scale_dic; /* :1135-1136 */
  free(v2);
  free(gdic);
  free(losses);
  return lossVal;
}

void orc_weight_gradient_scale(int W, int H, int D, double gamma, int P, int K, int L,
                               int loss_type, int log_domain, double scale_dic, const double* x,
                               const double* obs, double* gw_scale, int nthreads) {
  const size_t N = (size_t)W * H * D, KN = (size_t)K * N, PK = (size_t)P * K;
  double* w = xalloc(PK);
  double* a = xalloc(KN);
  for (size_t i = 0; i < PK; ++i) w[i] = exp(x[i] / scale_dic);
  for (size_t i = 0; i < KN; ++i) a[i] = exp(x[PK + i]);
  for (int p = 0; p < P; ++p) {
    double s = 0;
    for (int k = 0; k < K; ++k) s += w[p * K + k];
    for (int k = 0; k < K; ++k) w[p * K + k] /= s;
  }
  for (int k = 0; k < K; ++k) {
    double s = 0;
    for (size_t j = 0; j < N; ++j) s += a[k * N + j];
    for (size_t j = 0; j < N; ++j) a[k * N + j] /= s;
  }
#ifdef _OPENMP
  if (nthreads < 1) nthreads = 1;
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
#endif
  for (int p = 0; p < P; ++p) {
    double la_abs[64];
    orc_gradient_both_scale(W, H, D, gamma, K, L, loss_type, log_domain, a, w + (size_t)p * K,
                            obs + (size_t)p * N, la_abs);
    double m = 0;
    for (int k = 0; k < K; ++k) m += w[p * K + k] * la_abs[k];
    for (int k = 0; k < K; ++k) gw_scale[p * K + k] = (la_abs[k] + m) * w[p * K + k] / scale_dic;
  }
  free(w);
  free(a);
}
