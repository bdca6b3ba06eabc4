"""GPU: the tensor-core operator beyond one 128-row tile and in 3-D.

Grids with a side above 128 (the reference's bundled images are 272 x 240 and
224 x 224) and 3-D grids run the split-BF16 / TF32 operator as tcgen05 axis
passes (one GEMM per axis, any side up to 512).  Checked against the FP64
oracle at the tensor-core operator tolerances of the 128-tile operator, and a
whole evaluate_both at the split-BF16 targets (barycenter 1e-4, gradients
1e-3)."""
import numpy as np
import pytest

from conftest import rel, rel_scaled

pytestmark = pytest.mark.gpu

TC_OP_TOL = {"tf32": 3e-3, "split_bf16": 2e-5}


def _kern(gamma, W, H, D, precision):
    from wassersteindictionarylearning_b200 import CudaGaussian2DKernel, CudaGaussian3DKernel
    if D > 1:
        return CudaGaussian3DKernel(gamma, W, H, D, precision=precision)
    return CudaGaussian2DKernel(gamma, W, H, precision=precision)


@pytest.mark.parametrize("shape", [(272, 240, 1), (224, 224, 1), (129, 200, 1), (512, 66, 1),
                                   (301, 131, 1), (48, 48, 48), (40, 33, 20), (130, 7, 9)])
def test_operator_beyond_one_tile(oracle, shape):
    W, H, D = shape
    N = W * H * D
    rng = np.random.default_rng(W * 7 + H * 3 + D)
    u = rng.random(2 * N)
    gamma = 9.0
    ref = oracle.convolve(W, H, D, gamma, u, 2)
    for precision, tol in TC_OP_TOL.items():
        k = _kern(gamma, W, H, D, precision)
        out = k.convolve(u, 2)
        out2 = k.convolve(u, 2)  # a second call on the same context
        assert rel(out, ref) < tol, precision
        assert np.array_equal(out, out2), precision
        k.close()


@pytest.mark.parametrize("shape", [(200, 152, 1), (24, 20, 16)])
def test_split_bf16_evaluate_beyond_one_tile(oracle, shape):
    from wassersteindictionarylearning_b200 import Problem, WassersteinRegression
    from wassersteindictionarylearning_b200.synthetic import make_problem, to_variables
    W, H, D = shape
    P, K, L, gamma, loss = 2, 3, 8, 6.0, 2
    cfg, obs, atoms, w = make_problem(None, seed=4, P=P, W=W, H=H, D=D, K=K, L=L, gamma=gamma,
                                      loss=loss)
    x = to_variables(w, atoms, cfg["scale_dic"])
    sd = cfg["scale_dic"]
    f_ref, g_ref, bary_ref = oracle.evaluate_both(W, H, D, gamma, P, K, L, loss, sd, x, obs,
                                                  want_bary=True)
    k = _kern(gamma, W, H, D, "split_bf16")
    reg = WassersteinRegression(Problem(np.ones((K, W * H * D)), obs, k, None, P), L, loss, sd)
    fv, g = reg.evaluate_both(x)
    assert rel(reg.last_barycenters, bary_ref) < 1e-4
    assert abs(fv - f_ref) <= 1e-4 * abs(f_ref)
    PK = P * K
    assert rel(g[PK:], g_ref[PK:]) < 1e-3
    scale = oracle.weight_gradient_scale(W, H, D, gamma, P, K, L, loss, sd, x, obs)
    assert rel_scaled(g[:PK], g_ref[:PK], scale) < 1e-3
    k.close()


@pytest.mark.parametrize("shape", [(272, 240, 1), (129, 200, 1), (40, 33, 20)])
@pytest.mark.parametrize("precision", ["split_bf16", "tf32"])
def test_axis_tile_heights_agree(shape, precision):
    """The axis pass has two tile heights (128 image rows, one CTA per SM; 64
    rows, two CTAs per SM) and two ways of staging its operands (the CTA's own
    loads, or TMA / bulk copies on a stage ring where the row pitch allows),
    and a persistent form that keeps the factor slab resident in SMEM, chosen per
    shape by timing every variant on the call's own data.  All issue
    the same MMAs on the same operand values for every output element (same K
    chunks in the same order), so the tuned context returns exactly what a
    context held at the default returns; the tuning call's result is the last
    variant's (the copy-engine form where it applies)."""
    import ctypes as C

    from wassersteindictionarylearning_b200._lib import check, lib
    W, H, D = shape
    N = W * H * D
    u = np.random.default_rng(11).random(6 * N)
    tuned = _kern(5.0, W, H, D, precision)
    plain = _kern(5.0, W, H, D, precision)
    check(lib().wdl_set_profiling(plain.ctx, 1), plain.ctx)  # profiling keeps the default height
    first = tuned.convolve(u, 6)   # times both heights
    again = tuned.convolve(u, 6)   # the chosen height
    ref = plain.convolve(u, 6)
    assert np.array_equal(first, ref) and np.array_equal(again, ref)
    n = lib().wdl_autotune_count(tuned.ctx)
    key, choice, ms = (C.c_longlong * 6)(), C.c_int(), C.c_float()
    heights = []
    for i in range(n):
        check(lib().wdl_autotune_entry(tuned.ctx, i, key, C.byref(choice), C.byref(ms)), tuned.ctx)
        if key[0] == 2:
            # tile height 64 or 128, plus 1000 for the copy-engine (TMA) staged form;
            # 2064 the persistent form with the factor slab resident in SMEM
            assert choice.value in (64, 128, 1064, 1128, 2064) and ms.value > 0
            heights.append(choice.value)
    assert len(heights) == (2 if D == 1 else 3)  # one entry per axis-pass shape
    assert lib().wdl_autotune_count(plain.ctx) == 0
    tuned.close()
    plain.close()
