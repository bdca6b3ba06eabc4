"""Test infrastructure only: ctypes bindings to the CPU oracles.

Two libraries, both checkers and never part of the product path:

* ``RefLib`` — the reference's own code (WassersteinDictionaryLearning
  ``cpp/*.h`` + ``cpp/lbfgs/lbfgs.c``) compiled unmodified by ``oracle/Makefile``
  into ``oracle/_ref/``.  It pins the restatement below and serves as the timed
  CPU baseline (``kind: "reference"``).
* ``OracleLib`` — ``oracle/wdl_oracle.c``, a plain-C FP64 restatement of the
  same algorithm (file:line citations inside).  It travels with the repository
  and is what GPU tests compare against when the reference build is absent.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU legs import
this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
BUILD_DIR = os.path.join(HERE, "_build")

_dp = C.POINTER(C.c_double)
_ucp = C.POINTER(C.c_ubyte)


def _p(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"], (a.dtype, a.flags)
    return a.ctypes.data_as(_dp)


def _u(a):
    assert a.dtype == np.uint8 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_ucp)


def build(quiet: bool = True) -> None:
    """Build the oracle libraries (the reference part only where its sources exist)."""
    out = subprocess.run(["make", "-C", HERE, "all"], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)
    if not quiet:
        print(out.stdout)


def ref_available() -> bool:
    return os.path.exists(os.path.join(REF_DIR, "libwdlref.so")) and os.path.exists(
        os.path.join(REF_DIR, "libwdlref_log.so"))


class OracleLib:
    """The C restatement (oracle/wdl_oracle.c)."""

    def __init__(self):
        path = os.path.join(BUILD_DIR, "libwdl_oracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        self.L = L
        L.orc_convolve.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, _dp, _dp, C.c_int]
        L.orc_log_convolve.argtypes = [C.c_int, C.c_int, C.c_double, _dp, _dp, C.c_int]
        L.orc_log_convolve_signed.argtypes = [C.c_int, C.c_int, C.c_double, _dp, _ucp, _dp, C.c_int]
        L.orc_loss.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, _dp, _dp, _dp]
        L.orc_loss.restype = C.c_double
        L.orc_gradient_both.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_int, C.c_int,
                                        C.c_int, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp]
        L.orc_gradient_both_log.argtypes = [C.c_int, C.c_int, C.c_double, C.c_int, C.c_int,
                                            C.c_int, _dp, _dp, _dp, _dp, _dp, _dp]
        L.orc_barycenter.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_int, C.c_int,
                                     _dp, _dp, _dp]
        L.orc_barycenter_log.argtypes = [C.c_int, C.c_int, C.c_double, C.c_int, C.c_int,
                                         _dp, _dp, _dp]
        L.orc_evaluate_both.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_int, C.c_int,
                                        C.c_int, C.c_int, C.c_int, C.c_double, _dp, _dp, _dp,
                                        _dp, _dp, _dp, C.c_int]
        L.orc_evaluate_both.restype = C.c_double
        L.orc_gradient_both_scale.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_int,
                                              C.c_int, C.c_int, C.c_int, _dp, _dp, _dp, _dp]
        L.orc_weight_gradient_scale.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_int,
                                                C.c_int, C.c_int, C.c_int, C.c_int, C.c_double,
                                                _dp, _dp, _dp, C.c_int]

    def convolve(self, W, H, D, gamma, u, nv):
        u = np.ascontiguousarray(u, dtype=np.float64)
        out = np.empty_like(u)
        self.L.orc_convolve(W, H, D, gamma, _p(u), _p(out), nv)
        return out

    def log_convolve(self, W, H, gamma, u, nv):
        u = np.ascontiguousarray(u, dtype=np.float64)
        out = np.empty_like(u)
        self.L.orc_log_convolve(W, H, gamma, _p(u), _p(out), nv)
        return out

    def log_convolve_signed(self, W, H, gamma, u, signs, nv):
        u = np.ascontiguousarray(u, dtype=np.float64)
        signs = np.ascontiguousarray(signs, dtype=np.uint8).copy()
        out = np.empty_like(u)
        self.L.orc_log_convolve_signed(W, H, gamma, _p(u), _u(signs), _p(out), nv)
        return out, signs

    def loss(self, loss_type, W, H, D, gamma, v1, v2):
        v1 = np.ascontiguousarray(v1, dtype=np.float64)
        v2 = np.ascontiguousarray(v2, dtype=np.float64)
        g = np.empty_like(v1)
        f = self.L.orc_loss(loss_type, W, H, D, gamma, _p(v1), _p(v2), _p(g))
        return f, g

    def gradient_both(self, W, H, D, gamma, K, L, loss_type, atoms, lambdas, obs, b_init=None,
                      want_b_last=False):
        N = W * H * D
        atoms = np.ascontiguousarray(atoms, dtype=np.float64)
        lambdas = np.ascontiguousarray(lambdas, dtype=np.float64)
        obs = np.ascontiguousarray(obs, dtype=np.float64)
        la = np.zeros(K)
        dic = np.zeros(K * N)
        bary = np.zeros(N)
        b_last = np.zeros(K * N) if want_b_last else None
        bi = None if b_init is None else np.ascontiguousarray(b_init, dtype=np.float64)
        self.L.orc_gradient_both(W, H, D, gamma, K, L, loss_type, _p(atoms), _p(lambdas), _p(obs),
                                 _p(bi), _p(la), _p(dic), _p(bary), _p(b_last))
        if want_b_last:
            return la, dic, bary, b_last
        return la, dic, bary

    def gradient_both_scale(self, W, H, D, gamma, K, L, loss_type, atoms, lambdas, obs,
                            log_domain=False):
        """Mass of the terms summed into resultLa (its floating-point condition scale)."""
        atoms = np.ascontiguousarray(atoms, dtype=np.float64)
        lambdas = np.ascontiguousarray(lambdas, dtype=np.float64)
        obs = np.ascontiguousarray(obs, dtype=np.float64)
        out = np.zeros(K)
        self.L.orc_gradient_both_scale(W, H, D, gamma, K, L, loss_type, int(log_domain), _p(atoms),
                                       _p(lambdas), _p(obs), _p(out))
        return out

    def weight_gradient_scale(self, W, H, D, gamma, P, K, L, loss_type, scale_dic, x, obs,
                              log_domain=False, nthreads=None):
        """Per-entry error scale of evaluate_both's weight gradient (see wdl_oracle.h)."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        obs = np.ascontiguousarray(obs, dtype=np.float64)
        out = np.zeros(P * K)
        self.L.orc_weight_gradient_scale(W, H, D, gamma, P, K, L, loss_type, int(log_domain),
                                         scale_dic, _p(x), _p(obs), _p(out),
                                         nthreads or os.cpu_count() or 1)
        return out

    def gradient_both_log(self, W, H, gamma, K, L, loss_type, atoms, lambdas, obs):
        N = W * H
        atoms = np.ascontiguousarray(atoms, dtype=np.float64)
        lambdas = np.ascontiguousarray(lambdas, dtype=np.float64)
        obs = np.ascontiguousarray(obs, dtype=np.float64)
        la = np.zeros(K)
        dic = np.zeros(K * N)
        bary = np.zeros(N)
        self.L.orc_gradient_both_log(W, H, gamma, K, L, loss_type, _p(atoms), _p(lambdas),
                                     _p(obs), _p(la), _p(dic), _p(bary))
        return la, dic, bary

    def barycenter(self, W, H, D, gamma, K, L, atoms, lambdas, log_domain=False):
        N = W * H * D
        atoms = np.ascontiguousarray(atoms, dtype=np.float64)
        lambdas = np.ascontiguousarray(lambdas, dtype=np.float64)
        bary = np.zeros(N)
        if log_domain:
            self.L.orc_barycenter_log(W, H, gamma, K, L, _p(atoms), _p(lambdas), _p(bary))
        else:
            self.L.orc_barycenter(W, H, D, gamma, K, L, _p(atoms), _p(lambdas), _p(bary))
        return bary

    def evaluate_both(self, W, H, D, gamma, P, K, L, loss_type, scale_dic, x, obs, log_domain=False,
                      b_storage=None, want_b_last=False, want_bary=False, nthreads=None):
        N = W * H * D
        x = np.ascontiguousarray(x, dtype=np.float64)
        obs = np.ascontiguousarray(obs, dtype=np.float64)
        g = np.zeros_like(x)
        bs = None if b_storage is None else np.ascontiguousarray(b_storage, dtype=np.float64)
        bl = np.zeros(P * K * N) if want_b_last else None
        bo = np.zeros(P * N) if want_bary else None
        nthreads = nthreads or os.cpu_count() or 1
        f = self.L.orc_evaluate_both(W, H, D, gamma, P, K, L, loss_type, int(log_domain), scale_dic,
                                     _p(x), _p(g), _p(obs), _p(bs), _p(bl), _p(bo), nthreads)
        out = [f, g]
        if want_b_last:
            out.append(bl)
        if want_bary:
            out.append(bo)
        return tuple(out)


class RefLib:
    """The reference's own implementation (oracle/_ref)."""

    def __init__(self):
        if not ref_available():
            build()
        self.K = C.CDLL(os.path.join(REF_DIR, "libwdlref.so"))
        self.G = C.CDLL(os.path.join(REF_DIR, "libwdlref_log.so"))
        K, G = self.K, self.G
        K.ref_convolve2d.argtypes = [C.c_int, C.c_double, C.c_int, C.c_int, _dp, _dp, C.c_int]
        K.ref_convolve3d.argtypes = [C.c_double, C.c_int, C.c_int, C.c_int, _dp, _dp, C.c_int]
        K.ref_gradient_both.argtypes = [C.c_int, C.c_double, C.c_int, C.c_int, C.c_int, C.c_int,
                                        C.c_int, C.c_int, _dp, _dp, _dp, _dp, _dp, _dp]
        K.ref_barycenter.argtypes = [C.c_int, C.c_double, C.c_int, C.c_int, C.c_int, C.c_int,
                                     C.c_int, _dp, _dp, _dp]
        K.ref_evaluate_both.argtypes = [C.c_int, C.c_double, C.c_int, C.c_int, C.c_int, C.c_int,
                                        C.c_int, C.c_int, C.c_int, C.c_double, _dp, _dp, _dp, C.c_int]
        K.ref_evaluate_both.restype = C.c_double
        K.ref_evaluate_both_warm.argtypes = [C.c_int, C.c_double, C.c_int, C.c_int, C.c_int,
                                             C.c_int, C.c_int, C.c_int, C.c_double, _dp, _dp, _dp,
                                             _dp, _dp, C.c_int]
        K.ref_evaluate_both_warm.restype = C.c_double
        K.ref_regress_both.argtypes = [C.c_double, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                       C.c_int, C.c_double, C.c_int, _dp, _dp, C.c_int]
        K.ref_loss.argtypes = [C.c_int, C.c_double, C.c_int, C.c_int, _dp, _dp, _dp]
        K.ref_loss.restype = C.c_double
        G.ref_log_convolve2d.argtypes = [C.c_double, C.c_int, C.c_int, _dp, _dp, C.c_int]
        G.ref_log_convolve2d_signed.argtypes = [C.c_double, C.c_int, C.c_int, _dp, _ucp, _dp, C.c_int]
        G.ref_gradient_both_log.argtypes = [C.c_double, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                            _dp, _dp, _dp, _dp, _dp, _dp]
        G.ref_barycenter_log.argtypes = [C.c_double, C.c_int, C.c_int, C.c_int, C.c_int, _dp, _dp, _dp]
        G.ref_evaluate_both_log.argtypes = [C.c_double, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                            C.c_int, C.c_double, _dp, _dp, _dp, C.c_int]
        G.ref_evaluate_both_log.restype = C.c_double

    def omp_threads(self) -> int:
        return self.K.ref_omp_threads()

    def convolve(self, W, H, D, gamma, u, nv, sse=False):
        u = np.ascontiguousarray(u, dtype=np.float64)
        out = np.empty_like(u)
        if D == 1:
            self.K.ref_convolve2d(int(sse), gamma, W, H, _p(u), _p(out), nv)
        else:
            self.K.ref_convolve3d(gamma, W, H, D, _p(u), _p(out), nv)
        return out

    def log_convolve(self, W, H, gamma, u, nv):
        u = np.ascontiguousarray(u, dtype=np.float64)
        out = np.empty_like(u)
        self.G.ref_log_convolve2d(gamma, W, H, _p(u), _p(out), nv)
        return out

    def log_convolve_signed(self, W, H, gamma, u, signs, nv):
        u = np.ascontiguousarray(u, dtype=np.float64)
        signs = np.ascontiguousarray(signs, dtype=np.uint8).copy()
        out = np.empty_like(u)
        self.G.ref_log_convolve2d_signed(gamma, W, H, _p(u), _u(signs), _p(out), nv)
        return out, signs

    def loss(self, loss_type, W, H, gamma, v1, v2):
        v1 = np.ascontiguousarray(v1, dtype=np.float64)
        v2 = np.ascontiguousarray(v2, dtype=np.float64)
        g = np.empty_like(v1)
        f = self.K.ref_loss(loss_type, gamma, W, H, _p(v1), _p(v2), _p(g))
        return f, g

    def gradient_both(self, W, H, D, gamma, K, L, loss_type, atoms, lambdas, obs, kind=None):
        N = W * H * D
        kind = (2 if D > 1 else 0) if kind is None else kind
        atoms = np.ascontiguousarray(atoms, dtype=np.float64)
        lambdas = np.ascontiguousarray(lambdas, dtype=np.float64)
        obs = np.ascontiguousarray(obs, dtype=np.float64)
        la, dic, bary = np.zeros(K), np.zeros(K * N), np.zeros(N)
        self.K.ref_gradient_both(kind, gamma, W, H, D, K, L, loss_type, _p(atoms), _p(lambdas),
                                 _p(obs), _p(la), _p(dic), _p(bary))
        return la, dic, bary

    def gradient_both_scale(self, W, H, D, gamma, K, L, loss_type, atoms, lambdas, obs,
                            log_domain=False):
        """Mass of the terms summed into resultLa (its floating-point condition scale)."""
        atoms = np.ascontiguousarray(atoms, dtype=np.float64)
        lambdas = np.ascontiguousarray(lambdas, dtype=np.float64)
        obs = np.ascontiguousarray(obs, dtype=np.float64)
        out = np.zeros(K)
        self.L.orc_gradient_both_scale(W, H, D, gamma, K, L, loss_type, int(log_domain), _p(atoms),
                                       _p(lambdas), _p(obs), _p(out))
        return out

    def weight_gradient_scale(self, W, H, D, gamma, P, K, L, loss_type, scale_dic, x, obs,
                              log_domain=False, nthreads=None):
        """Per-entry error scale of evaluate_both's weight gradient (see wdl_oracle.h)."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        obs = np.ascontiguousarray(obs, dtype=np.float64)
        out = np.zeros(P * K)
        self.L.orc_weight_gradient_scale(W, H, D, gamma, P, K, L, loss_type, int(log_domain),
                                         scale_dic, _p(x), _p(obs), _p(out),
                                         nthreads or os.cpu_count() or 1)
        return out

    def gradient_both_log(self, W, H, gamma, K, L, loss_type, atoms, lambdas, obs):
        N = W * H
        atoms = np.ascontiguousarray(atoms, dtype=np.float64)
        lambdas = np.ascontiguousarray(lambdas, dtype=np.float64)
        obs = np.ascontiguousarray(obs, dtype=np.float64)
        la, dic, bary = np.zeros(K), np.zeros(K * N), np.zeros(N)
        self.G.ref_gradient_both_log(gamma, W, H, K, L, loss_type, _p(atoms), _p(lambdas),
                                     _p(obs), _p(la), _p(dic), _p(bary))
        return la, dic, bary

    def barycenter(self, W, H, D, gamma, K, L, atoms, lambdas, log_domain=False):
        N = W * H * D
        atoms = np.ascontiguousarray(atoms, dtype=np.float64)
        lambdas = np.ascontiguousarray(lambdas, dtype=np.float64)
        bary = np.zeros(N)
        if log_domain:
            self.G.ref_barycenter_log(gamma, W, H, K, L, _p(atoms), _p(lambdas), _p(bary))
        else:
            self.K.ref_barycenter(2 if D > 1 else 0, gamma, W, H, D, K, L, _p(atoms), _p(lambdas),
                                  _p(bary))
        return bary

    def evaluate_both(self, W, H, D, gamma, P, K, L, loss_type, scale_dic, x, obs,
                      log_domain=False, kind=None, quiet=True):
        x = np.ascontiguousarray(x, dtype=np.float64)
        obs = np.ascontiguousarray(obs, dtype=np.float64)
        g = np.zeros_like(x)
        if log_domain:
            f = self.G.ref_evaluate_both_log(gamma, W, H, P, K, L, loss_type, scale_dic, _p(x),
                                             _p(g), _p(obs), int(quiet))
        else:
            kind = (2 if D > 1 else 0) if kind is None else kind
            f = self.K.ref_evaluate_both(kind, gamma, W, H, D, P, K, L, loss_type, scale_dic,
                                         _p(x), _p(g), _p(obs), int(quiet))
        return f, g

    def evaluate_both_warm(self, W, H, gamma, P, K, L, loss_type, scale_dic, x, obs, b_storage,
                           quiet=True):
        x = np.ascontiguousarray(x, dtype=np.float64)
        obs = np.ascontiguousarray(obs, dtype=np.float64)
        bs = np.ascontiguousarray(b_storage, dtype=np.float64)
        g = np.zeros_like(x)
        bl = np.zeros_like(bs)
        f = self.K.ref_evaluate_both_warm(0, gamma, W, H, P, K, L, loss_type, scale_dic, _p(x),
                                          _p(g), _p(obs), _p(bs), _p(bl), int(quiet))
        return f, g, bl

    def regress_both(self, W, H, gamma, P, K, L, loss_type, scale_dic, max_iter, solution, obs,
                     quiet=True):
        sol = np.ascontiguousarray(solution, dtype=np.float64).copy()
        obs = np.ascontiguousarray(obs, dtype=np.float64)
        self.K.ref_regress_both(gamma, W, H, P, K, L, loss_type, scale_dic, max_iter, _p(sol),
                                _p(obs), int(quiet))
        return sol
