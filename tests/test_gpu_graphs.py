"""GPU: the CUDA-core evaluation path replays repeated calls as a CUDA graph.

A call with the same sizes, buffers and stream as an earlier one is captured
once and replayed; the replay must produce exactly what the eager launches
produce (the CUDA-core path is deterministic), for new input values too, and
count the same kernel launches."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _grad(kern, atoms, w, obs, K, L, loss=2):
    from wassersteindictionarylearning_b200._lib import check, dptr, lib
    P = w.shape[0]
    N = kern.N if hasattr(kern, "N") else atoms.shape[1]
    la, dic, bary, f = np.empty(P * K), np.empty(K * N), np.empty(P * N), np.empty(P)
    check(lib().wdl_gradient_both(kern.ctx, P, K, L, loss, dptr(atoms), dptr(w), dptr(obs), None,
                                  dptr(la), dptr(dic), dptr(bary), dptr(f), None), kern.ctx)
    return la, dic, bary, f


@pytest.mark.parametrize("kind", ["kernel_fp32", "log_fp32", "kernel_fp64"])
def test_graph_replay_is_bitwise_eager(kind):
    from wassersteindictionarylearning_b200 import (CudaGaussian2DKernel,
                                                    CudaLogSignArrayGaussian2DKernel)
    from wassersteindictionarylearning_b200._lib import lib
    from wassersteindictionarylearning_b200.synthetic import blob_histograms, init_weights
    W, H, K, L, P, gamma = 24, 20, 3, 6, 2, 2.0
    prec = "fp64" if kind.endswith("fp64") else "fp32"
    make = CudaLogSignArrayGaussian2DKernel if kind.startswith("log") else CudaGaussian2DKernel
    atoms = blob_histograms(K, W, H, seed=1) + 1.0 / (W * H)
    obs = blob_histograms(P, W, H, seed=2)
    wA, wB = init_weights(P, K, seed=3), init_weights(P, K, seed=4)
    kern = make(gamma, W, H, precision=prec)
    ref = make(gamma, W, H, precision=prec)
    lib().wdl_set_profiling(ref.ctx, 1)  # profiling keeps every call eager
    eA, eB = _grad(ref, atoms, wA, obs, K, L), _grad(ref, atoms, wB, obs, K, L)
    r1 = _grad(kern, atoms, wA, obs, K, L)          # eager (the first call also autotunes)
    n1 = lib().wdl_launch_count(kern.ctx)
    r2 = _grad(kern, atoms, wA, obs, K, L)          # captured, then launched
    n2 = lib().wdl_launch_count(kern.ctx)
    r3 = _grad(kern, atoms, wB, obs, K, L)          # replay, new inputs
    r4 = _grad(kern, atoms, wA, obs, K, L)          # replay
    n4 = lib().wdl_launch_count(kern.ctx)
    for a, b in [(r1, eA), (r2, eA), (r3, eB), (r4, eA)]:
        for x, y in zip(a, b):
            assert np.array_equal(x, y)
    assert n4 - n2 == 2 * (n2 - n1) > 0
    kern.close()
    ref.close()


def test_autotuned_log_pass_is_bitwise_default():
    """The autotuner times every rows-per-block variant of the log-domain axis
    pass on a call's own data and keeps the fastest; the variants compute each
    output with the same operations, so results never depend on the choice."""
    from wassersteindictionarylearning_b200 import CudaLogSignArrayGaussian2DKernel
    from wassersteindictionarylearning_b200._lib import check, dptr, lib
    W, H, nv = 96, 80, 6
    rng = np.random.default_rng(0)
    u = np.log(rng.random(nv * W * H) + 1e-3) * 40.0
    tuned = CudaLogSignArrayGaussian2DKernel(0.7, W, H, precision="fp32")
    plain = CudaLogSignArrayGaussian2DKernel(0.7, W, H, precision="fp32")
    lib().wdl_set_profiling(plain.ctx, 1)  # profiling keeps the default variant
    outs = []
    for kern in (tuned, tuned, plain):
        o = np.empty_like(u)
        check(lib().wdl_log_convolve(kern.ctx, dptr(u), dptr(o), nv), kern.ctx)
        outs.append(o)
    # the tuning call's result is the last candidate's (32 rows per block)
    assert np.array_equal(outs[0], outs[2]) and np.array_equal(outs[1], outs[2])
    # the signed operator likewise, values and signs
    signs0 = np.random.default_rng(1).integers(0, 256, (nv * W * H + 7) // 8).astype(np.uint8)
    souts = []
    for kern in (tuned, tuned, plain):
        sg = signs0.copy()
        o = np.empty_like(u)
        check(lib().wdl_log_convolve_signed(kern.ctx, dptr(u), sg.ctypes.data_as(C.POINTER(C.c_ubyte)),
                                            dptr(o), nv), kern.ctx)
        souts.append((o, sg))
    for o, sg in souts[:2]:
        assert np.array_equal(o, souts[2][0]) and np.array_equal(sg, souts[2][1])
    n = lib().wdl_autotune_count(tuned.ctx)
    assert n >= 2  # one entry per axis pass shape
    key, choice, ms = (C.c_longlong * 6)(), C.c_int(), C.c_float()
    for i in range(n):
        check(lib().wdl_autotune_entry(tuned.ctx, i, key, C.byref(choice), C.byref(ms)), tuned.ctx)
        # rows per block
        assert key[0] == 1 and choice.value in (8, 16, 32) and ms.value > 0
    assert lib().wdl_autotune_count(plain.ctx) == 0
    tuned.close()
    plain.close()
