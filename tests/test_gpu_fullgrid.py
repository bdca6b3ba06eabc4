"""GPU parity on full grids: the log-domain configuration's 256x256 grid (K=8,
gamma 0.5, TV loss, sharp blobs) and the serving volume 48^3 (K=5, L=50) against
the reference's own outputs.

The fixtures (tests/golden/full_*.npz, written by make_golden.py --large from
the reference build) hold no inputs: they are regenerated here from the
recorded seeds and checked against the stored input statistics first.  Large
outputs are stored as every STRIDE-th entry plus the whole array's maximum
magnitude, sum and sum of magnitudes; the comparisons are normwise
(max|a - b| / max|b|) over the stored entries and relative on the whole-array
sums, with the tolerances of the other parity tests: FP64 1e-10, FP32 1e-5.
Weight gradients are measured against their condition scale (stored with the
fixture), as in test_gpu_parity.py.

The log-domain operator skips taps whose terms lie 40 bits (FP32) or 60 nats
(FP64) below the running maximum and takes the FP32 logarithm from lg2.approx:
these grids, where most taps are cut, are where that shows if it matters.
"""
import numpy as np
import pytest

from conftest import golden, rel, rel_scaled

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-10, "fp32": 1e-5}


def _inputs_match(f, *arrays):
    stats = np.array([v for a in arrays for v in (float(np.sum(a)), float(np.sum(np.asarray(a) ** 2)),
                                                  float(np.max(a)), float(np.min(a)))])
    assert np.allclose(stats, f["in_stats"], rtol=1e-12, atol=0), "regenerated inputs differ"


def _check_sampled(f, prefix, a, tol):
    a = np.asarray(a, dtype=np.float64).reshape(-1)
    stride = int(f[prefix + "_stride"])
    assert a.size == int(f[prefix + "_n"])
    ref = f[prefix + "_sample"]
    absmax = float(f[prefix + "_absmax"])
    assert float(np.max(np.abs(a[::stride] - ref))) / absmax < tol
    assert abs(float(np.max(np.abs(a))) - absmax) / absmax < tol
    assert abs(float(np.sum(np.abs(a))) - float(f[prefix + "_abssum"])) / float(f[prefix + "_abssum"]) < tol
    # the signed sum against the mass of its terms
    assert abs(float(np.sum(a)) - float(f[prefix + "_total"])) / float(f[prefix + "_abssum"]) < tol


def _one(pattern):
    (name, f), = golden(pattern)
    return f


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_log256_gradient_both(precision):
    """compute_gradient_both_log_signArray (cpp/inverseWasserstein.h:678-814) at 256x256."""
    from wassersteindictionarylearning_b200 import (CudaLogSignArrayGaussian2DKernel, Problem,
                                                     WassersteinRegression)
    from wassersteindictionarylearning_b200.synthetic import blob_histograms, init_atoms, init_weights
    f = _one("full_gradlog_256x256_*")
    W, H, K, L, g, lt = (int(f["W"]), int(f["H"]), int(f["K"]), int(f["L"]), float(f["gamma"]),
                         int(f["loss"]))
    s_obs, s_atoms, s_lam = (int(v) for v in f["seeds"])
    obs = blob_histograms(1, W, H, n_blobs=(1, 3), std_frac=(0.01, 0.04), seed=s_obs)[0]
    atoms = init_atoms(K, W * H, seed=s_atoms)
    lam = init_weights(1, K, seed=s_lam)[0]
    _inputs_match(f, obs, atoms, lam)
    k = CudaLogSignArrayGaussian2DKernel(g, W, H, precision=precision)
    reg = WassersteinRegression(Problem(np.ones((K, W * H)), obs, k, None, 1), L, lt, 1.0)
    la, dic, bary, loss = reg.compute_gradient_both(atoms, lam)
    tol = TOL[precision]
    assert rel(bary, f["bary"]) < tol
    # TV loss of the barycenter (cpp/loss.h:19-40) against the reference's barycenter
    loss_ref = 0.5 * float(np.sum(np.abs(f["bary"] - obs)))
    assert abs(float(np.ravel(loss)[0]) - loss_ref) / loss_ref < tol
    _check_sampled(f, "resultDic", dic, tol)
    assert rel_scaled(la, f["resultLa"], f["resultLa_scale"]) < tol


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_log256_evaluate_both(precision):
    """evaluate_both (cpp/inverseWasserstein.h:986-1145) in the log domain, P=2, 256x256."""
    from wassersteindictionarylearning_b200 import (CudaLogSignArrayGaussian2DKernel, Problem,
                                                     WassersteinRegression)
    from wassersteindictionarylearning_b200.synthetic import (blob_histograms, init_atoms, init_weights,
                                                              to_variables)
    f = _one("full_eval_P2_256x256_*")
    P, W, H, K, L, g, lt = (int(f["P"]), int(f["W"]), int(f["H"]), int(f["K"]), int(f["L"]),
                            float(f["gamma"]), int(f["loss"]))
    sd = float(f["scale_dic"])
    s_obs, s_atoms, s_w = (int(v) for v in f["seeds"])
    obs = blob_histograms(P, W, H, n_blobs=(1, 3), std_frac=(0.01, 0.04), seed=s_obs)
    atoms = init_atoms(K, W * H, seed=s_atoms)
    w = init_weights(P, K, seed=s_w)
    _inputs_match(f, obs, atoms, w)
    x = to_variables(w, atoms, sd)
    k = CudaLogSignArrayGaussian2DKernel(g, W, H, precision=precision)
    reg = WassersteinRegression(Problem(np.ones((K, W * H)), obs, k, None, P), L, lt, sd)
    fv, grad = reg.evaluate_both(x)
    tol = TOL[precision]
    assert abs(fv - float(f["f"])) <= tol * abs(float(f["f"]))
    _check_sampled(f, "g_atoms", grad[P * K:], tol)
    assert rel_scaled(grad[:P * K], f["g_weights"], f["g_weights_scale"]) < tol


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_log256_signed_operator(precision):
    """log_convolve and log_convolve_signArray (cpp/kernels.h:1073-1163) at 256x256, gamma 0.5."""
    from wassersteindictionarylearning_b200 import CudaLogSignArrayGaussian2DKernel
    f = _one("full_logconv_256x256_*")
    W, H, g = int(f["W"]), int(f["H"]), float(f["gamma"])
    rng = np.random.Generator(np.random.PCG64(int(f["seed"])))
    u = np.log(rng.random(W * H)) * 3.0
    signs = rng.integers(0, 256, (W * H + 7) // 8).astype(np.uint8)
    _inputs_match(f, u)
    assert np.array_equal(signs, f["signs_in"])
    k = CudaLogSignArrayGaussian2DKernel(g, W, H, precision=precision)
    tol = 1e-13 if precision == "fp64" else 1e-5
    _check_sampled(f, "out", k.log_convolve(u, 1), tol)
    out = k.log_convolve_signArray(u, signs, 1)
    # A signed sum S = sum_k s_k t_k cancels: any summation order's error in
    # log|S| is up to (taps * eps) * cond with cond = sum_k t_k / |S|, and
    # exp(unsigned output - signed output) is that cond (up to 8.9e4 here).
    stride = int(f["out_signed_stride"])
    cond = np.exp(f["out_sample"] - f["out_signed_sample"])
    err = np.abs(out[::stride] - f["out_signed_sample"])
    per_cond = 1e-12 if precision == "fp64" else 1e-4  # 256 taps x eps, with margin
    assert np.all(err <= per_cond * np.maximum(cond, 1.0)), float(np.max(err / np.maximum(cond, 1.0)))
    same = np.unpackbits(signs, bitorder="little")[: W * H] == \
        np.unpackbits(f["signs_out"], bitorder="little")[: W * H]
    if precision == "fp64":
        assert same.all()
    else:  # near-cancelling signed sums may flip in FP32
        assert same.mean() > 0.97


@pytest.mark.parametrize("precision", ["fp64", "fp32", "split_bf16"])
def test_volume48_gradient_both(precision):
    """compute_gradient_both (cpp/inverseWasserstein.h:544-674) with Gaussian3DKernel on the
    serving volume 48^3, K=5, L=50, gamma 2, in the kernel domain."""
    from wassersteindictionarylearning_b200 import (CudaGaussian3DKernel, Problem,
                                                     WassersteinRegression)
    from wassersteindictionarylearning_b200.synthetic import blob_histograms, init_atoms, init_weights
    f = _one("full_grad_48x48x48_*")
    W, H, D, K, L = (int(f[k]) for k in ("W", "H", "D", "K", "L"))
    g, lt = float(f["gamma"]), int(f["loss"])
    s_obs, s_atoms, s_lam = (int(v) for v in f["seeds"])
    obs = blob_histograms(1, W, H, D, n_blobs=(1, 3), std_frac=(0.05, 0.12), seed=s_obs)[0]
    atoms = init_atoms(K, W * H * D, seed=s_atoms)
    lam = init_weights(1, K, seed=s_lam)[0]
    _inputs_match(f, obs, atoms, lam)
    k = CudaGaussian3DKernel(g, W, H, D, precision=precision)
    reg = WassersteinRegression(Problem(np.ones((K, W * H * D)), obs, k, None, 1), L, lt, 1.0)
    la, dic, bary, _ = reg.compute_gradient_both(atoms, lam)
    # split-BF16: the north star's targets against FP64 (barycenter 1e-4, gradients 1e-3)
    tol_b, tol_g = (1e-4, 1e-3) if precision == "split_bf16" else (TOL[precision],) * 2
    _check_sampled(f, "bary", bary, tol_b)
    _check_sampled(f, "resultDic", dic, tol_g)
    assert rel_scaled(la, f["resultLa"], f["resultLa_scale"]) < tol_g
