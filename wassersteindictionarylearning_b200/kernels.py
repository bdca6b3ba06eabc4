"""CUDA KernelType objects: Python mirror of the reference's kernel classes.

``CudaGaussian2DKernel(gamma, W, H)`` stands where ``Gaussian2DKernel`` /
``GaussianSSE2DKernel`` stand (cpp/kernels.h:630-907), ``CudaGaussian3DKernel``
for ``Gaussian3DKernel`` (:712-815), and ``CudaLogSignArrayGaussian2DKernel`` for
``LogSignArrayGaussian2DKernel`` (:1034-1202).  Each owns a device context of
libwdl_b200; ``convolve``/``convolveAdjoint``/``log_convolve*`` take and return
float64 arrays of ``nvectors`` stacked images exactly like the reference's
members (with the output returned instead of written through a pointer).
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _lib
from ._lib import check, dptr, f64, lib

EPSILON = 1e-250  # cpp/kernels.h:30


class _CudaKernelBase:
    """Shared context management; ``precision`` is one of fp32/tf32/split_bf16/fp64."""

    def __init__(self, gamma: float, W: int, H: int, D: int, precision: str, domain: int,
                 device: int = -1):
        self.gamma = float(gamma)
        self.W_, self.H_, self.D_ = int(W), int(H), int(D)
        self.N = self.W_ * self.H_ * self.D_
        self.precision = precision
        self.domain = domain
        h = C.c_void_p()
        check(lib().wdl_create(C.byref(h), device, self.W_, self.H_, self.D_, self.gamma,
                               _lib.PRECISIONS[precision], domain))
        self._ctx = h

    @property
    def ctx(self):
        return self._ctx

    def close(self):
        if getattr(self, "_ctx", None) is not None and self._ctx.value:
            lib().wdl_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __call__(self, i: int, j: int) -> float:
        """Kernel matrix entry (operator(), cpp/kernels.h:660-667)."""
        W, H = self.W_, self.H_
        zi, zj = i // (W * H), j // (W * H)
        i, j = i - zi * W * H, j - zj * W * H
        d2 = (i % W - j % W) ** 2 + (i // W - j // W) ** 2 + (zi - zj) ** 2
        return max(EPSILON, math.exp(-d2 / self.gamma))

    def convolve(self, u, nvectors: int = 1) -> np.ndarray:
        u = f64(u).reshape(-1)
        assert u.size == nvectors * self.N
        out = np.empty_like(u)
        check(lib().wdl_convolve(self._ctx, dptr(u), dptr(out), nvectors), self._ctx)
        return out

    def convolveAdjoint(self, u, nvectors: int = 1) -> np.ndarray:
        return self.convolve(u, nvectors)


class CudaGaussian2DKernel(_CudaKernelBase):
    def __init__(self, gamma: float = 25.0, W: int = 0, H: int = 0, precision: str = "fp32",
                 device: int = -1):
        super().__init__(gamma, W, H, 1, precision, _lib.WDL_DOMAIN_KERNEL, device)


class CudaGaussian3DKernel(_CudaKernelBase):
    def __init__(self, gamma: float = 25.0, W: int = 0, H: int = 0, D: int = 0,
                 precision: str = "fp32", device: int = -1):
        super().__init__(gamma, W, H, D, precision, _lib.WDL_DOMAIN_KERNEL, device)


class CudaLogSignArrayGaussian2DKernel(_CudaKernelBase):
    def __init__(self, gamma: float = 25.0, W: int = 0, H: int = 0, precision: str = "fp32",
                 device: int = -1):
        super().__init__(gamma, W, H, 1, precision, _lib.WDL_DOMAIN_LOG, device)

    def log_convolve(self, log_u, nvectors: int = 1) -> np.ndarray:
        u = f64(log_u).reshape(-1)
        out = np.empty_like(u)
        check(lib().wdl_log_convolve(self._ctx, dptr(u), dptr(out), nvectors), self._ctx)
        return out

    def log_convolveAdjoint(self, log_u, nvectors: int = 1) -> np.ndarray:
        return self.log_convolve(log_u, nvectors)

    def log_convolve_signArray(self, log_u, sign_array: np.ndarray, nvectors: int = 1):
        """Signed log-sum-exp; ``sign_array`` (uint8, bit-packed, bit=1 means >= 0) is
        read for the input and overwritten in place with the output's signs."""
        u = f64(log_u).reshape(-1)
        assert sign_array.dtype == np.uint8 and sign_array.flags["C_CONTIGUOUS"]
        out = np.empty_like(u)
        check(lib().wdl_log_convolve_signed(self._ctx, dptr(u),
                                            sign_array.ctypes.data_as(C.POINTER(C.c_ubyte)),
                                            dptr(out), nvectors), self._ctx)
        return out

    def log_convolve_signArrayAdjoint(self, log_u, sign_array, nvectors: int = 1):
        return self.log_convolve_signArray(log_u, sign_array, nvectors)
