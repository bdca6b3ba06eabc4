"""GPU: the no-allocation operator entry point (wdl_convolve_device_noalloc).

Some callers cannot allocate device memory once they run (hosts that reserve
all memory at start-up, processes under a device-memory cap or pool).  For them
the library offers the operator with its scratch in a fixed array compiled into
the library, reserved on the device when a context is created.  This test calls
it through the C ABI and checks it against the regular entry point
(wdl_convolve_device) with the tolerances of the operator tests, on two calls in
a row (the shared scratch keeps the previous call's contents); checks that the
device's free memory is the same before and after a first call on a new
context and grid; and checks that an oversized request is refused.  It lives in
its own file, collected last.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import rel

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-13, "fp32": 1e-6, "split_bf16": 1e-6}


@pytest.mark.parametrize("precision", ["fp64", "fp32", "split_bf16"])
def test_noalloc_matches_regular_entry_point(precision):
    import torch

    from wassersteindictionarylearning_b200 import CudaGaussian2DKernel, _lib
    L = _lib.lib()
    W, H, nv = 96, 80, 5
    k = CudaGaussian2DKernel(1.5, W, H, precision=precision, device=0)
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(device=dev)
    rng = np.random.default_rng(7)
    u = torch.from_numpy(rng.random(nv * W * H)).to(dev)
    ref = torch.empty_like(u)
    out1 = torch.empty_like(u)
    out2 = torch.empty_like(u)
    sp = C.c_void_p(stream.cuda_stream)
    _lib.check(L.wdl_convolve_device(k.ctx, C.c_void_p(u.data_ptr()), C.c_void_p(ref.data_ptr()),
                                     nv, sp), k.ctx)
    for out in (out1, out2):
        _lib.check(L.wdl_convolve_device_noalloc(k.ctx, C.c_void_p(u.data_ptr()),
                                                 C.c_void_p(out.data_ptr()), nv, sp), k.ctx)
    stream.synchronize()
    r = ref.cpu().numpy()
    assert rel(out1.cpu().numpy(), r) < TOL[precision]
    assert rel(out2.cpu().numpy(), r) < TOL[precision]


def test_noalloc_call_allocates_nothing():
    import torch

    from wassersteindictionarylearning_b200 import CudaGaussian2DKernel, _lib
    L = _lib.lib()
    dev = torch.device("cuda", 0)

    def call(k, u, out, nv):
        _lib.check(L.wdl_convolve_device_noalloc(k.ctx, C.c_void_p(u.data_ptr()),
                                                 C.c_void_p(out.data_ptr()), nv, None), k.ctx)
        _lib.check(L.wdl_synchronize(k.ctx), k.ctx)

    # one call on another grid first, so that the kernels' code is loaded (CUDA
    # loads a kernel on its first launch in the process)
    warm = CudaGaussian2DKernel(2.0, 40, 24, precision="fp32", device=0)
    wu = torch.ones(40 * 24, dtype=torch.float64, device=dev)
    call(warm, wu, torch.empty_like(wu), 1)

    W, H, nv = 72, 56, 3
    u = torch.from_numpy(np.random.default_rng(3).random(nv * W * H)).to(dev)
    out = torch.empty_like(u)
    ref = torch.empty_like(u)
    k = CudaGaussian2DKernel(2.0, W, H, precision="fp32", device=0)  # fresh context: empty arena
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(dev)
    call(k, u, out, nv)
    free1, _ = torch.cuda.mem_get_info(dev)
    assert free1 == free0, (free0, free1)
    _lib.check(L.wdl_convolve_device(k.ctx, C.c_void_p(u.data_ptr()), C.c_void_p(ref.data_ptr()), nv,
                                     None), k.ctx)
    _lib.check(L.wdl_synchronize(k.ctx), k.ctx)
    assert rel(out.cpu().numpy(), ref.cpu().numpy()) < TOL["fp32"]


def test_noalloc_rejects_oversized_request():
    import torch

    from wassersteindictionarylearning_b200 import CudaGaussian2DKernel, _lib
    L = _lib.lib()
    k = CudaGaussian2DKernel(1.0, 128, 128, precision="fp64", device=0)
    big = 200  # 3 * 200 * 16384 * 8 bytes > 32 MiB
    buf = torch.zeros(1, dtype=torch.float64, device="cuda:0")
    rc = L.wdl_convolve_device_noalloc(k.ctx, C.c_void_p(buf.data_ptr()), C.c_void_p(buf.data_ptr()),
                                       big, None)
    assert rc == -1
    assert b"scratch" in L.wdl_last_error(k.ctx)
