"""GPU: the batched and fitting entry points refuse what they cannot do with
a status and a message, before launching anything."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _fit_problem(W=16, H=16, K=3, L=4, P=1, loss=2):
    from wassersteindictionarylearning_b200._lib import WdlFitProblem, dptr
    N = W * H
    keep = dict(a=np.full(K * N, 1.0 / N), o=np.full(P * N, 1.0 / N), w=np.empty(P * K),
                f=np.empty(P), st=np.empty(P, dtype=np.int32), ev=np.empty(P, dtype=np.int32))
    fp = WdlFitProblem(W, H, K, L, P, loss, dptr(keep["a"]), dptr(keep["o"]), None, dptr(keep["w"]),
                       dptr(keep["f"]), keep["st"].ctypes.data_as(C.POINTER(C.c_int)),
                       keep["ev"].ctypes.data_as(C.POINTER(C.c_int)))
    return fp, keep


def test_fit_entry_points_validate():
    from wassersteindictionarylearning_b200 import CudaGaussian2DKernel, CudaLogSignArrayGaussian2DKernel
    from wassersteindictionarylearning_b200._lib import lib
    L_ = lib()
    kern = CudaGaussian2DKernel(2.0, 64, 64, precision="split_bf16")
    logk = CudaLogSignArrayGaussian2DKernel(2.0, 64, 64, precision="fp32")
    fp, keep = _fit_problem()
    arr = (type(fp) * 1)(fp)
    # the log-domain fit wants a log-domain context, the kernel-domain fit a kernel one
    assert L_.wdl_fit_weights_log(kern.ctx, C.cast(arr, C.c_void_p), 1, 5, 1e-6) == -4
    assert b"log-domain" in L_.wdl_last_error(kern.ctx)
    assert L_.wdl_fit_weights(logk.ctx, C.cast(arr, C.c_void_p), 1, 5, 1e-6) == -4
    # K above the log fit's limit, a loss it does not take, negative iteration counts
    fp_big, keep2 = _fit_problem(K=17)
    arr2 = (type(fp) * 1)(fp_big)
    assert L_.wdl_fit_weights_log(logk.ctx, C.cast(arr2, C.c_void_p), 1, 5, 1e-6) == -1
    fp_w, keep3 = _fit_problem(loss=3)
    arr3 = (type(fp) * 1)(fp_w)
    assert L_.wdl_fit_weights_log(logk.ctx, C.cast(arr3, C.c_void_p), 1, 5, 1e-6) == -1
    assert L_.wdl_fit_weights(kern.ctx, C.cast(arr, C.c_void_p), 1, -1, 1e-6) == -1
    assert L_.wdl_fit_weights_log(logk.ctx, C.cast(arr, C.c_void_p), 0, 5, 1e-6) == -1
    kern.close()
    logk.close()


def test_batch_run_validates():
    from wassersteindictionarylearning_b200 import CudaGaussian2DKernel
    from wassersteindictionarylearning_b200._lib import WdlProblem, dptr, lib
    L_ = lib()
    kern = CudaGaussian2DKernel(2.0, 64, 64, precision="split_bf16")
    W = 80  # above the context's side
    a, w, o = np.full(3 * W * W, 1.0), np.full(3, 1.0 / 3), np.full(W * W, 1.0)
    la, f = np.empty(3), np.empty(1)
    pb = (WdlProblem * 1)(WdlProblem(W, W, 3, 4, 1, 2, 0, dptr(a), dptr(w), dptr(o), dptr(la), None,
                                     None, dptr(f)))
    assert L_.wdl_batch_run(kern.ctx, C.cast(pb, C.c_void_p), 1) == -1
    # a context beyond the fused kernel's 128 tile has no many-problem launch
    big = CudaGaussian2DKernel(2.0, 200, 160, precision="split_bf16")
    assert L_.wdl_batch_run(big.ctx, C.cast(pb, C.c_void_p), 1) == -4
    kern.close()
    big.close()


def test_tensor_core_context_limits():
    from wassersteindictionarylearning_b200._lib import lib
    ctx = C.c_void_p()
    # sides up to 512 take the tensor-core precisions; beyond, creation fails
    assert lib().wdl_create(C.byref(ctx), 0, 600, 64, 1, 2.0, 2, 0) == -4
    assert lib().wdl_create(C.byref(ctx), 0, 512, 64, 1, 2.0, 2, 0) == 0
    lib().wdl_destroy(ctx)
