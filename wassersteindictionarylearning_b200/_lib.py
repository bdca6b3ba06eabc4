"""ctypes binding of libwdl_b200.so (the C ABI of include/wdl.h).

The library is built in-tree (``make -C wassersteindictionarylearning_b200``) and
loaded from ``wassersteindictionarylearning_b200/lib/``.  There is no fallback:
if the library is missing or no sm_100 device is present, calls raise.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "lib", "libwdl_b200.so")

WDL_OK = 0
WDL_FP32, WDL_TF32, WDL_SPLIT_BF16, WDL_FP64 = 0, 1, 2, 3
WDL_DOMAIN_KERNEL, WDL_DOMAIN_LOG = 0, 1
PRECISIONS = {"fp32": WDL_FP32, "tf32": WDL_TF32, "split_bf16": WDL_SPLIT_BF16, "fp64": WDL_FP64}

ERRORS = {
    -1: "WDL_ERR_INVALID_ARG", -2: "WDL_ERR_CUDA", -3: "WDL_ERR_OUT_OF_MEMORY",
    -4: "WDL_ERR_UNSUPPORTED", -5: "WDL_ERR_NONFINITE", -6: "WDL_ERR_TIMEOUT",
    -7: "WDL_ERR_ADMISSION", -8: "WDL_ERR_NO_DEVICE", -9: "WDL_ERR_BUSY",
}

_dp = C.POINTER(C.c_double)
_vp = C.c_void_p

WDL_MODE_WEIGHTS, WDL_MODE_BOTH, WDL_MODE_BARYCENTER = 0, 1, 2
WDL_FIT_OVERFLOW = -2000
WDL_FAULT_DROP_FIRST_ITERATION = 1


class WdlProblem(C.Structure):
    """struct wdl_problem of include/wdl.h."""
    _fields_ = [("W", C.c_int), ("H", C.c_int), ("K", C.c_int), ("L", C.c_int), ("P", C.c_int),
                ("loss_type", C.c_int), ("mode", C.c_int), ("atoms", _dp), ("weights", _dp),
                ("observed", _dp), ("result_la", _dp), ("result_dic", _dp), ("bary", _dp),
                ("loss", _dp)]


class WdlFitProblem(C.Structure):
    """struct wdl_fit_problem of include/wdl.h."""
    _fields_ = [("W", C.c_int), ("H", C.c_int), ("K", C.c_int), ("L", C.c_int), ("P", C.c_int),
                ("loss_type", C.c_int), ("atoms", _dp), ("observed", _dp), ("x0", _dp),
                ("weights", _dp), ("loss", _dp), ("status", C.POINTER(C.c_int)),
                ("evaluations", C.POINTER(C.c_int))]


class WdlError(RuntimeError):
    def __init__(self, code: int, detail: str):
        self.code = code
        super().__init__(f"{ERRORS.get(code, code)}: {detail}")


def build(quiet: bool = True) -> None:
    """Compile the CUDA library in-tree for sm_100a (nvcc cross-compiles without a GPU)."""
    out = subprocess.run(["make", "-C", PKG, "-j8"], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("libwdl_b200 build failed:\n" + out.stdout[-4000:] + out.stderr[-8000:])
    if not quiet:
        print(out.stdout)


# Every symbol include/wdl.h declares, with its ctypes signature.
SIGNATURES = {
    "wdl_abi_version": ([], C.c_int),
    "wdl_strerror": ([C.c_int], C.c_char_p),
    "wdl_last_error": ([_vp], C.c_char_p),
    "wdl_create": ([C.POINTER(_vp), C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_int,
                    C.c_int], C.c_int),
    "wdl_destroy": ([_vp], C.c_int),
    "wdl_synchronize": ([_vp], C.c_int),
    "wdl_eval_bytes": ([_vp, C.c_int, C.c_int, C.c_int], C.c_size_t),
    "wdl_convolve": ([_vp, _dp, _dp, C.c_int], C.c_int),
    "wdl_log_convolve": ([_vp, _dp, _dp, C.c_int], C.c_int),
    "wdl_log_convolve_signed": ([_vp, _dp, C.POINTER(C.c_ubyte), _dp, C.c_int], C.c_int),
    "wdl_gradient_both": ([_vp, C.c_int, C.c_int, C.c_int, C.c_int, _dp, _dp, _dp, _dp, _dp, _dp,
                           _dp, _dp, _dp], C.c_int),
    "wdl_evaluate_both": ([_vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, _dp, _dp, C.c_int,
                           _dp, _dp, _dp, _dp, _dp], C.c_int),
    "wdl_barycenter": ([_vp, C.c_int, C.c_int, C.c_int, _dp, _dp, _dp], C.c_int),
    "wdl_evaluate_both_device": ([_vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, _vp, _vp,
                                  C.c_int, _vp, _vp, _vp, _vp, _vp, _vp], C.c_int),
    "wdl_gradient_both_device": ([_vp, C.c_int, C.c_int, C.c_int, C.c_int, _vp, _vp, _vp, _vp, _vp,
                                  _vp, _vp, _vp, _vp, _vp], C.c_int),
    "wdl_convolve_device": ([_vp, _vp, _vp, C.c_int, _vp], C.c_int),
    "wdl_convolve_device_noalloc": ([_vp, _vp, _vp, C.c_int, _vp], C.c_int),
    "wdl_batch_run": ([_vp, C.c_void_p, C.c_int], C.c_int),
    "wdl_fit_weights": ([_vp, C.c_void_p, C.c_int, C.c_int, C.c_double], C.c_int),
    "wdl_fit_weights_log": ([_vp, C.c_void_p, C.c_int, C.c_int, C.c_double], C.c_int),
    "wdl_fit_weights_operator": ([_vp, C.c_int, C.c_int, C.c_int, C.c_int, _dp, _dp, _dp, C.c_int,
                                  C.c_double, _dp, _dp, C.POINTER(C.c_int), C.POINTER(C.c_int)], C.c_int),
    "wdl_launch_count": ([_vp], C.c_longlong),
    "wdl_set_profiling": ([_vp, C.c_int], C.c_int),
    "wdl_conv_profile": ([_vp, _dp, C.POINTER(C.c_longlong), _dp], C.c_int),
    "wdl_phase_trace": ([_vp, _dp], C.c_int),
    "wdl_exp_profile": ([_vp, _dp], C.c_int),
    "wdl_set_autotune": ([_vp, C.c_int], C.c_int),
    "wdl_set_wait_limit": ([_vp, C.c_double], C.c_int),
    "wdl_regress_both": ([_vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, _dp, _dp, C.c_int,
                          C.c_double, C.c_int, C.POINTER(C.c_int), _dp, C.POINTER(C.c_int)], C.c_int),
    "wdl_regress_both_device": ([_vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, _vp, _vp, C.c_int,
                                 C.c_double, C.c_int, C.POINTER(C.c_int), _dp, C.POINTER(C.c_int), _vp],
                                C.c_int),
    "wdl_inject_fault": ([_vp, C.c_int], C.c_int),
    "wdl_autotune_count": ([_vp], C.c_int),
    "wdl_autotune_entry": ([_vp, C.c_int, C.POINTER(C.c_longlong), C.POINTER(C.c_int),
                            C.POINTER(C.c_float)], C.c_int),
}

_LIB = None


def lib():
    """Load the library once; raise with the build hint if it is absent."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: run `make -C {PKG}` (nvcc, sm_100a)")
        L = C.CDLL(LIB_PATH)
        for name, (args, res) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _LIB = L
    return _LIB


def check(rc: int, ctx=None) -> None:
    if rc != WDL_OK:
        detail = lib().wdl_last_error(ctx)
        raise WdlError(rc, detail.decode() if detail else "")


def dptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_dp)


def f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)
