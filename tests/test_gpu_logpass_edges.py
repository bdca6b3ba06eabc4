"""GPU: the log-domain operator (log_convolve, log_convolve_signArray;
cpp/kernels.h:1073-1163) at the grid edges its axis pass treats specially.

The pass makes four neighbouring outputs of a row per thread and stages rows
with a halo of 8 taps, so the cases worth pinning against the oracle are: rows
shorter than one group or not a multiple of 4 (partial groups), rows shorter
than the halo, and wide kernels or spread-out inputs whose taps reach past
the halo (the range-tested steps).  Unsigned results in every case, signed ones
checked against the signed sum's condition number (a cancelling sum's log
carries the summation error times that condition in any order)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SHAPES = [(1, 5), (2, 3), (3, 7), (5, 1), (7, 9), (13, 6), (33, 17), (4, 64)]


def _inputs(W, H, nv, spread, seed):
    rng = np.random.default_rng(seed)
    u = np.log(rng.random(W * H * nv) + 1e-12) * spread
    signs = rng.integers(0, 256, (W * H * nv + 7) // 8).astype(np.uint8)
    return u, signs


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("gamma,spread", [(0.3, 5.0), (4.0, 5.0), (60.0, 5.0), (0.7, 60.0)])
@pytest.mark.parametrize("W,H", SHAPES)
def test_log_operator_edges(oracle, W, H, gamma, spread, precision):
    from wassersteindictionarylearning_b200 import CudaLogSignArrayGaussian2DKernel
    nv = 3
    u, signs = _inputs(W, H, nv, spread, seed=W * 100 + H)
    k = CudaLogSignArrayGaussian2DKernel(gamma, W, H, precision=precision)
    tol = 1e-12 if precision == "fp64" else 2e-6
    ref = oracle.log_convolve(W, H, gamma, u, nv)
    out = k.log_convolve(u, nv)
    err = np.abs(out - ref)
    assert np.all(err <= tol * np.maximum(1.0, np.abs(ref))), float(np.max(err / np.maximum(1.0, np.abs(ref))))

    ref_s, sg_ref = oracle.log_convolve_signed(W, H, gamma, u, signs, nv)
    sg = signs.copy()
    out_s = k.log_convolve_signArray(u, sg, nv)
    # cond = sum of the terms' magnitudes / |signed sum| = exp(unsigned - signed)
    cond = np.exp(np.minimum(ref - ref_s, 700.0))
    err_s = np.abs(out_s - ref_s)
    bound = 50 * tol * np.maximum(1.0, np.abs(ref)) * np.maximum(cond, 1.0)
    finite = np.isfinite(ref_s)
    assert np.all(err_s[finite] <= bound[finite]), float(np.max((err_s / bound)[finite]))
    same = np.unpackbits(sg, bitorder="little")[: W * H * nv] == \
        np.unpackbits(sg_ref, bitorder="little")[: W * H * nv]
    if precision == "fp64":
        assert same[cond < 1e6].all()
    else:  # the first pass's signed sums may cancel too; FP32 can flip those
        assert same[cond < 1e2].mean() > 0.99
    k.close()
