"""GPU: a bounded wait of the fused tensor-core kernel running out.

The fault is made on the host (wdl_inject_fault): the work table of one
wdl_batch_run call leaves out the first forward iteration, so every other item
waits on a completion flag that nothing publishes.  With the dependency-wait
bound shortened to 50 ms, the call must return WDL_ERR_TIMEOUT well within a
second or two (the kernel's items stop and it exits normally: no trap, no
unbounded wait), and the same context must then run a normal batch whose
results equal those of a fresh context.  The reference's analogue is the
NaN-loss cancel of L-BFGS (cpp/inverseWasserstein.h:1180-1184).
"""
import time

import numpy as np
import pytest

from conftest import rel

pytestmark = pytest.mark.gpu

WDL_ERR_TIMEOUT = -6


def _problems():
    from wassersteindictionarylearning_b200.synthetic import blob_histograms, init_weights
    W, H, K, L, P = 32, 32, 3, 6, 2
    return [dict(W=W, H=H, K=K, L=L, P=P, mode="both", loss_type=2, want_bary=True,
                 atoms=blob_histograms(K, W, H, seed=5).reshape(-1),
                 weights=init_weights(P, K, seed=6).reshape(-1),
                 observed=blob_histograms(P, W, H, seed=7).reshape(-1))]


def test_dependency_wait_runs_out_and_context_recovers():
    from wassersteindictionarylearning_b200 import CudaGaussian2DKernel, _lib
    from wassersteindictionarylearning_b200.batch import batch_run
    L = _lib.lib()
    probs = _problems()
    k = CudaGaussian2DKernel(1.5, 64, 64, precision="split_bf16", device=0)
    ref = batch_run(CudaGaussian2DKernel(1.5, 64, 64, precision="split_bf16", device=0), probs)

    assert L.wdl_set_wait_limit(k.ctx, 0.05) == 0
    assert L.wdl_inject_fault(k.ctx, _lib.WDL_FAULT_DROP_FIRST_ITERATION) == 0
    t0 = time.perf_counter()
    with pytest.raises(RuntimeError) as err:
        batch_run(k, probs)
    elapsed = time.perf_counter() - t0
    assert err.value.code == WDL_ERR_TIMEOUT, str(err.value)
    assert elapsed < 2.0, elapsed

    # the context is still usable: default bound, no fault, the results of a fresh
    # context (the fused kernel's float atomics make repeated runs agree to the
    # split-BF16 rounding, not bitwise: barycenter and loss 1e-4, gradients 1e-3)
    assert L.wdl_set_wait_limit(k.ctx, 0.0) == 0
    out = batch_run(k, probs)
    for key, tol in (("bary", 1e-4), ("loss", 1e-4), ("la", 1e-3), ("dic", 1e-3)):
        assert rel(out[0][key], ref[0][key]) < tol, key


def test_wait_limit_arguments():
    from wassersteindictionarylearning_b200 import CudaGaussian2DKernel, _lib
    L = _lib.lib()
    k = CudaGaussian2DKernel(1.0, 16, 16, precision="split_bf16", device=0)
    assert L.wdl_set_wait_limit(k.ctx, -1.0) == -1
    assert L.wdl_set_wait_limit(k.ctx, 61.0) == -1
    assert L.wdl_inject_fault(k.ctx, 7) == -1
    assert L.wdl_inject_fault(k.ctx, 0) == 0
