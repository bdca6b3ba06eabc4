/* Test infrastructure only — the CPU oracle for the Sinkhorn-barycenter hot path.
 *
 * A plain-C FP64 restatement of the reference's algorithm
 * (WassersteinDictionaryLearning: cpp/kernels.h, cpp/inverseWasserstein.h,
 * cpp/loss.h).  Only tests/, __graft_entry__.smoke() and bench.py's CPU arms
 * may load it, and only as the checker or the timed CPU baseline; the product
 * library never calls it.  It is pinned against the reference itself
 * (oracle/_ref, built from the reference sources) by tests/test_oracle.py and
 * by the golden fixtures in tests/golden/.
 *
 * Layout conventions follow the reference: images are row-major
 * (x fastest, index y*W+x; 3-D: z*W*H + y*W + x), K images of N=W*H*D pixels
 * are stacked with stride N, and the optimisation vector is
 * x = [P*K scaled log-weights, K*N log-atoms] (main_dictionary_learning.cpp:139-159).
 * D = 1 selects the 2-D operator.
 */
#ifndef WDL_ORACLE_H
#define WDL_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

#define ORC_EPSILON 1e-250 /* cpp/kernels.h:30 */

/* 1-D Gibbs factor max(EPSILON, exp(-i^2/gamma)), i = 0..n-1 (cpp/kernels.h:637-640). */
void orc_kernel1d(double gamma, int n, double* out);

/* Separable Gaussian on nv stacked images (cpp/kernels.h:669-699, 3-D :762-807). */
void orc_convolve(int W, int H, int D, double gamma, const double* u, double* out, int nv);

/* Stabilised log-sum-exp convolution, two-pass per output (cpp/kernels.h:1073-1112). */
void orc_log_convolve(int W, int H, double gamma, const double* log_u, double* out, int nv);

/* Signed variant: input signs read from `signs` (bit=1 means >= 0), output
 * signs written back into the same array (cpp/kernels.h:1117-1159). */
void orc_log_convolve_signed(int W, int H, double gamma, const double* log_u,
                             unsigned char* signs, double* out, int nv);

/* Loss value and gradient (cpp/loss.h:19-90).  loss_type 1=TV 2=quadratic 4=KL;
 * 3 (Wasserstein, cpp/loss.h:92-154) uses the kernel-domain operator of (W,H,D,gamma). */
double orc_loss(int loss_type, int W, int H, int D, double gamma, const double* v1,
                const double* v2, double* grad);

/* compute_gradient_both for one histogram (cpp/inverseWasserstein.h:544-674):
 * atoms/lambdas are normalised in place of a copy (normalize_values, :53-74).
 * b_init (K*N) or NULL for ones; b_last (K*N) or NULL receives b[L]. */
void orc_gradient_both(int W, int H, int D, double gamma, int K, int L, int loss_type,
                       const double* atoms, const double* lambdas, const double* obs,
                       const double* b_init, double* resultLa, double* resultDic,
                       double* bary, double* b_last);

/* Condition scale of resultLa: la_abs[k] = sum over steps s and pixels j of
 * |log(phi[s]_kj) g_j| (log domain: |phi g|), the mass of the terms whose sum is
 * resultLa[k].  A floating-point evaluation of resultLa is accurate to a small
 * multiple of unit roundoff times la_abs, not times |resultLa|, which can be far
 * smaller after cancellation.  Test infrastructure only. */
void orc_gradient_both_scale(int W, int H, int D, double gamma, int K, int L, int loss_type,
                             int log_domain, const double* atoms, const double* lambdas,
                             const double* obs, double* la_abs);

/* compute_gradient_both_log_signArray (cpp/inverseWasserstein.h:678-814). */
void orc_gradient_both_log(int W, int H, double gamma, int K, int L, int loss_type,
                           const double* atoms, const double* lambdas, const double* obs,
                           double* resultLa, double* resultDic, double* bary);

/* WassersteinBarycenter::compute_barycenter (cpp/inverseWasserstein.h:115-153)
 * and compute_barycenter_log (:155-201). */
void orc_barycenter(int W, int H, int D, double gamma, int K, int L, const double* atoms,
                    const double* lambdas, double* bary);
void orc_barycenter_log(int W, int H, double gamma, int K, int L, const double* atoms,
                        const double* lambdas, double* bary);

/* evaluate_both (cpp/inverseWasserstein.h:986-1145), exp_weight = true.
 * log_domain selects the log-domain histogram path.  b_storage (P*K*N) or NULL,
 * b_last (P*K*N) or NULL implement the warm restart carry (:1057-1061, :1081-1085).
 * bary_out (P*N) or NULL receives each histogram's barycenter.
 * Histograms are processed in parallel with OpenMP when nthreads > 1. */
double orc_evaluate_both(int W, int H, int D, double gamma, int P, int K, int L, int loss_type,
                         int log_domain, double scale_dic, const double* x, double* g,
                         const double* obs, const double* b_storage, double* b_last,
                         double* bary_out, int nthreads);

/* Condition scale of evaluate_both's weight gradient (test infrastructure):
 * gw_scale[p*K+k] = (la_abs_pk + sum_j w_pj la_abs_pj) * w_pk / scale_dic, the
 * error bound of g[p*K+k] = (la_pk - <w_p, la_p>) w_pk / scale_dic in units of
 * the relative error of the la terms. */
void orc_weight_gradient_scale(int W, int H, int D, double gamma, int P, int K, int L,
                               int loss_type, int log_domain, double scale_dic, const double* x,
                               const double* obs, double* gw_scale, int nthreads);

#ifdef __cplusplus
}
#endif
#endif
