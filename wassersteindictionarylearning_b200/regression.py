"""Problem / WassersteinBarycenter / WassersteinRegression over the CUDA path.

Mirrors the public surface of the reference's classes in
cpp/inverseWasserstein.h (Problem :29-95, WassersteinBarycenter :99-320,
WassersteinRegression :323-1230) with a CUDA KernelType: the per-histogram
loop of ``evaluate_both`` (:1052-1113) is one device call for all P
histograms, and ``regress_both`` (:362-521) drives it with the host L-BFGS of
``lbfgs.py`` using the reference's parameters (:365-372).
"""
from __future__ import annotations

import ctypes as C
import math
from typing import Optional

import numpy as np

from . import lbfgs as _lb
from ._lib import WdlError, check, dptr, f64, lib
from .kernels import _CudaKernelBase

LOSS_TV, LOSS_QUADRATIC, LOSS_WASSERSTEIN, LOSS_KL = 1, 2, 3, 4


class Problem:
    """Atoms pdfs[K][N], observed histograms [P*N], barycentric weights lambdas[K]."""

    def __init__(self, histograms, observed_histogram, kernel: _CudaKernelBase, weights=None,
                 npdfs: int = 1):
        self.pdfs = f64(histograms).reshape(-1, kernel.N).copy()
        self.K = self.pdfs.shape[0]
        self.N = kernel.N
        self.observed_pdf = f64(observed_histogram).reshape(-1).copy()
        self.kernel = kernel
        self.num_pdfs = npdfs
        self.lambdas = np.zeros(self.K) if weights is None else f64(weights)[: self.K].copy()

    def set_weights(self, weights):
        self.lambdas = f64(weights)[: self.K].copy()

    def set_pdfs(self, vertex_pdfs):
        self.pdfs = f64(vertex_pdfs).reshape(self.K, self.N).copy()

    def normalize_values(self):
        self.lambdas = self.lambdas / self.lambdas.sum()
        self.pdfs = self.pdfs / self.pdfs.sum(axis=1, keepdims=True)


class WassersteinBarycenter:
    """Forward Bregman projections for given weights (cpp/inverseWasserstein.h:99-320)."""

    def __init__(self, problem: Problem, n_bregman_iter: int):
        self.problem = problem
        self.K, self.N = problem.K, problem.N
        self.Niters = int(n_bregman_iter)
        self.barycenter = None

    def compute_barycenter(self, weights: Optional[np.ndarray] = None) -> np.ndarray:
        """Barycenter of the atoms for one weight vector (or P of them, shape (P, K))."""
        w = self.problem.lambdas if weights is None else f64(weights)
        w = np.atleast_2d(w)
        P = w.shape[0]
        out = np.empty(P * self.N)
        ctx = self.problem.kernel.ctx
        check(lib().wdl_barycenter(ctx, P, self.K, self.Niters, dptr(f64(self.problem.pdfs)),
                                   dptr(f64(w)), dptr(out)), ctx)
        self.barycenter = out if P > 1 else out.copy()
        return out.reshape(P, self.N) if P > 1 else out

    compute_barycenter_log = compute_barycenter

    def get_barycenter(self):
        return self.barycenter


class WassersteinRegression:
    """Dictionary learning objective and driver over the device path."""

    def __init__(self, problem: Problem, n_bregman_iterations: int, loss_type: int,
                 scale_dictionary: float = 0.0, warm_restart: bool = False):
        self.problem = problem
        self.K, self.N = problem.K, problem.N
        self.P = problem.num_pdfs
        self.Niters = int(n_bregman_iterations)
        self.loss_type = int(loss_type)
        self.scaleDictionary = float(scale_dictionary)
        self.warmRestart = bool(warm_restart)
        self.exp_weight = True
        self.wrTotalIteration = 0
        self.iteration = 0
        self.b_storage = None
        self.b_temp = None
        self.lbfgs_param = _lb.LbfgsParam(epsilon=1e-50, max_linesearch=20, delta=1e-50)
        self.last_barycenters = None
        self.verbose = False

    # ---- objective -------------------------------------------------------------
    def evaluate_both(self, x: np.ndarray, step: float = 0.0):
        """(f, g) at x = [P*K scaled log-weights, K*N log-atoms] (:986-1145)."""
        if not self.exp_weight:
            raise WdlError(-4, "exp_weight = false (allowNegWeights) is not supported")
        x = f64(x)
        n = x.size
        g = np.empty(n)
        fv = np.zeros(1)
        bary = np.empty(self.P * self.N)
        ctx = self.problem.kernel.ctx
        b_last = None
        if self.warmRestart:
            if self.b_storage is None:
                self.b_storage = np.ones(self.P * self.K * self.N)
            b_last = np.empty(self.P * self.K * self.N)
        rc = lib().wdl_evaluate_both(ctx, self.P, self.K, self.Niters, self.loss_type,
                                     self.scaleDictionary, dptr(x), dptr(g), n,
                                     dptr(self.problem.observed_pdf), dptr(fv),
                                     dptr(self.b_storage) if self.warmRestart else None,
                                     dptr(b_last), dptr(bary))
        if rc != -5:  # a non-finite objective is returned to L-BFGS, as the reference does
            check(rc, ctx)
        if self.warmRestart:
            self.b_temp = b_last
        self.last_barycenters = bary
        return float(fv[0]), g

    def compute_gradient_both(self, atoms, weights, b_init=None):
        """Raw resultLa [P*K], resultDic summed over P [K*N], barycenters [P*N] and
        per-histogram losses [P] for normalised inputs (:544-674 for all P at once)."""
        P, K, N = self.P, self.K, self.N
        la, dic = np.empty(P * K), np.empty(K * N)
        bary, loss = np.empty(P * N), np.empty(P)
        ctx = self.problem.kernel.ctx
        check(lib().wdl_gradient_both(ctx, P, K, self.Niters, self.loss_type, dptr(f64(atoms)),
                                      dptr(f64(weights)), dptr(self.problem.observed_pdf),
                                      dptr(None if b_init is None else f64(b_init)), dptr(la),
                                      dptr(dic), dptr(bary), dptr(loss), None), ctx)
        return la, dic, bary, loss

    # ---- driver ------------------------------------------------------------------
    def progress_both(self, x, g, fx, xnorm, gnorm, step, k, ls):
        self.iteration += 1
        if self.verbose:
            print(f"Iteration {k}: loss {fx:.12e} step {step:.3e}")
        if math.isnan(fx):  # :1180-1184
            return _lb.LBFGSERR_CANCELED
        return 0

    def regress_both_device(self, solution: np.ndarray) -> int:
        """regress_both with the L-BFGS on the device (wdl_regress_both): the
        same optimisation, no per-evaluation host round trip of the n-vectors.
        Optimises ``solution`` (original domain) in place; returns liblbfgs'
        status of the last run."""
        P, K, N = self.P, self.K, self.N
        sol = f64(solution)
        status, fval, evals = C.c_int(), C.c_double(), C.c_int()
        ctx = self.problem.kernel.ctx
        check(lib().wdl_regress_both(ctx, P, K, self.Niters, self.loss_type, self.scaleDictionary,
                                     dptr(sol), dptr(self.problem.observed_pdf), int(self.wrTotalIteration),
                                     float(self.lbfgs_param.epsilon), int(bool(self.warmRestart)),
                                     C.byref(status), C.byref(fval), C.byref(evals)), ctx)
        solution[:] = sol
        self.device_evaluations = evals.value
        self.device_objective = fval.value
        return status.value

    def regress_both(self, solution: np.ndarray) -> int:
        """Optimise [weights, atoms] in place (original domain on entry and exit)."""
        P, K, N = self.P, self.K, self.N
        sd = self.scaleDictionary
        sol = f64(solution)
        x = np.concatenate([np.log(sol[: P * K]) * sd, np.log(sol[P * K:])])
        self.iteration = 0
        runs = 1
        p = self.lbfgs_param
        if self.warmRestart:
            p.max_iterations = 10
            runs = self.wrTotalIteration // 10
            self.b_storage = np.ones(P * K * N)
        else:
            p.max_iterations = self.wrTotalIteration
        ret = 0
        for _ in range(runs):
            ret, x, _f = _lb.lbfgs(x, self.evaluate_both, self.progress_both, p)
            if self.warmRestart and self.b_temp is not None:
                self.b_storage = self.b_temp.copy()
        w = np.exp(x[: P * K] / sd).reshape(P, K)
        w /= w.sum(axis=1, keepdims=True)
        a = np.exp(x[P * K:]).reshape(K, N)
        a /= a.sum(axis=1, keepdims=True)
        solution[: P * K] = w.reshape(-1)
        solution[P * K:] = a.reshape(-1)
        return ret
