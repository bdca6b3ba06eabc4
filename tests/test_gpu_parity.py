"""GPU parity: the CUDA path (through the C ABI) against the reference's golden
outputs and the oracle.

Tolerances against the FP64 reference:
  FP64 mode   1e-10, FP32 mode 1e-5.
Barycenters, losses and the dictionary gradient use the normwise relative error
||x - ref||_inf / ||ref||_inf.  The weight gradients are differences of
near-equal sums (the per-step dot products of the reverse pass, then the simplex
projection), so their error is measured against the mass of the summed terms
(oracle.gradient_both_scale / weight_gradient_scale), the quantity that any
floating-point evaluation's error is proportional to.
"""
import numpy as np
import pytest

from conftest import golden, rel, rel_scaled

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-10, "fp32": 1e-5}


def kern(gamma, W, H, D=1, precision="fp64", log=False):
    from wassersteindictionarylearning_b200 import (CudaGaussian2DKernel, CudaGaussian3DKernel,
                                                     CudaLogSignArrayGaussian2DKernel)
    if log:
        return CudaLogSignArrayGaussian2DKernel(gamma, W, H, precision=precision)
    if D > 1:
        return CudaGaussian3DKernel(gamma, W, H, D, precision=precision)
    return CudaGaussian2DKernel(gamma, W, H, precision=precision)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("name,f", golden("conv_*"))
def test_convolve(name, f, precision):
    k = kern(float(f["gamma"]), int(f["W"]), int(f["H"]), int(f["D"]), precision)
    out = k.convolve(f["u"], int(f["nv"]))
    assert rel(out, f["out"]) < (1e-13 if precision == "fp64" else 1e-6)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("name,f", golden("logconv_*"))
def test_log_convolve(name, f, precision):
    W, H, nv = int(f["W"]), int(f["H"]), int(f["nv"])
    k = kern(float(f["gamma"]), W, H, precision=precision, log=True)
    tol = 1e-13 if precision == "fp64" else 1e-5
    assert rel(k.log_convolve(f["u"], nv), f["out"]) < tol
    signs = f["signs_in"].copy()
    out = k.log_convolve_signArray(f["u"], signs, nv)
    if precision == "fp64":
        assert np.array_equal(signs, f["signs_out"])
        assert rel(out, f["out_signed"]) < tol
    else:  # near-cancelling sums may flip; compare where the reference is far from 0
        ok = np.unpackbits(signs, bitorder="little")[: W * H * nv] == \
            np.unpackbits(f["signs_out"], bitorder="little")[: W * H * nv]
        assert ok.mean() > 0.97


def _regression(W, H, D, gamma, P, K, L, loss, sd, obs, precision, log=False):
    from wassersteindictionarylearning_b200 import Problem, WassersteinRegression
    k = kern(gamma, W, H, D, precision, log)
    prob = Problem(np.ones((K, W * H * D)), obs, k, None, P)
    return WassersteinRegression(prob, L, loss, sd)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("name,f", golden("grad_*"))
def test_gradient_both(oracle, name, f, precision):
    W, H, D, K, L = int(f["W"]), int(f["H"]), int(f["D"]), int(f["K"]), int(f["L"])
    reg = _regression(W, H, D, float(f["gamma"]), 1, K, L, int(f["loss"]), 1.0, f["obs"], precision)
    la, dic, bary, _ = reg.compute_gradient_both(f["atoms"], f["lambdas"])
    tol = TOL[precision]
    assert rel(bary, f["bary"]) < tol
    assert rel(dic, f["resultDic"]) < tol
    scale = oracle.gradient_both_scale(W, H, D, float(f["gamma"]), K, L, int(f["loss"]), f["atoms"],
                                       f["lambdas"], f["obs"])
    assert rel_scaled(la, f["resultLa"], scale) < tol


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("name,f", golden("gradlog_*"))
def test_gradient_both_log(oracle, name, f, precision):
    W, H, K, L = int(f["W"]), int(f["H"]), int(f["K"]), int(f["L"])
    reg = _regression(W, H, 1, float(f["gamma"]), 1, K, L, int(f["loss"]), 1.0, f["obs"], precision,
                      log=True)
    la, dic, bary, _ = reg.compute_gradient_both(f["atoms"], f["lambdas"])
    tol = TOL[precision]
    assert rel(bary, f["bary"]) < tol
    assert rel(dic, f["resultDic"]) < tol
    scale = oracle.gradient_both_scale(W, H, 1, float(f["gamma"]), K, L, int(f["loss"]), f["atoms"],
                                       f["lambdas"], f["obs"], log_domain=True)
    assert rel_scaled(la, f["resultLa"], scale) < tol


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("name,f", golden("bary_*"))
def test_barycenter(name, f, precision):
    from wassersteindictionarylearning_b200 import Problem, WassersteinBarycenter
    W, H, D, K, L = int(f["W"]), int(f["H"]), int(f["D"]), int(f["K"]), int(f["L"])
    k = kern(float(f["gamma"]), W, H, D, precision, log=bool(f["log"]))
    prob = Problem(f["atoms"], np.zeros(W * H * D), k, f["lambdas"], 1)
    b = WassersteinBarycenter(prob, L).compute_barycenter()
    assert rel(b, f["bary"]) < TOL[precision]


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("name,f", golden("eval_*"))
def test_evaluate_both(oracle, name, f, precision):
    W, H, D, P, K, L = (int(f[k]) for k in ("W", "H", "D", "P", "K", "L"))
    reg = _regression(W, H, D, float(f["gamma"]), P, K, L, int(f["loss"]), float(f["scale_dic"]),
                      f["obs"], precision, log=bool(f["log"]))
    fv, g = reg.evaluate_both(f["x"])
    tol = TOL[precision]
    assert abs(fv - float(f["f"])) <= tol * abs(float(f["f"]))
    check_gradient(oracle, g, f["g"], W, H, D, float(f["gamma"]), P, K, L, int(f["loss"]),
                   float(f["scale_dic"]), f["x"], f["obs"], tol, tol, log=bool(f["log"]))


def check_gradient(oracle, g, g_ref, W, H, D, gamma, P, K, L, loss, sd, x, obs, tol_w, tol_a,
                   log=False):
    """Atom part normwise; weight part against its condition scale."""
    PK = P * K
    assert rel(g[PK:], g_ref[PK:]) < tol_a
    scale = oracle.weight_gradient_scale(W, H, D, gamma, P, K, L, loss, sd, x, obs, log_domain=log)
    assert rel_scaled(g[:PK], g_ref[:PK], scale) < tol_w


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_warm_restart(precision):
    # (weights compared at 1e-3 normwise: the warm-started scalings make the
    # condition scale of the oracle's cold-start run inapplicable)
    (_, f), = golden("warm_*")
    W, H, P, K, L = (int(f[k]) for k in ("W", "H", "P", "K", "L"))
    reg = _regression(W, H, 1, float(f["gamma"]), P, K, L, int(f["loss"]), float(f["scale_dic"]),
                      f["obs"], precision)
    reg.warmRestart = True
    reg.b_storage = f["b_storage"].copy()
    fv, g = reg.evaluate_both(f["x"])
    tol = TOL[precision]
    assert abs(fv - float(f["f"])) <= tol * abs(float(f["f"]))
    assert rel(reg.b_temp, f["b_last"]) < tol
    PK = P * K
    assert rel(g[PK:], f["g"][PK:]) < tol
    assert rel(g[:PK], f["g"][:PK]) < 1e-3


def test_regress_both_matches_reference():
    """Four L-BFGS iterations end to end through the GPU (FP64) land where the
    reference's regress_both does."""
    (_, f), = golden("regress_*")
    W, H, P, K, L = (int(f[k]) for k in ("W", "H", "P", "K", "L"))
    reg = _regression(W, H, 1, float(f["gamma"]), P, K, L, int(f["loss"]), float(f["scale_dic"]),
                      f["obs"], "fp64")
    reg.wrTotalIteration = int(f["iters"])
    sol = f["solution0"].copy()
    reg.regress_both(sol)
    assert rel(sol, f["solution"]) < 1e-8


# ---- larger cases against the oracle -----------------------------------------------
def _problem(P, W, H, K, L, gamma, loss, D=1, seed=0, n_blobs=(1, 3)):
    from wassersteindictionarylearning_b200.synthetic import make_problem, to_variables
    cfg, obs, atoms, w = make_problem(None, seed=seed, P=P, W=W, H=H, D=D, K=K, L=L, gamma=gamma,
                                      loss=loss, n_blobs=n_blobs)
    x = to_variables(w, atoms, cfg["scale_dic"])
    return cfg, obs, x


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
@pytest.mark.parametrize("case", [
    dict(P=16, W=64, H=64, K=4, L=25, gamma=2.0, loss=2),            # dictionary-learning shape
    dict(P=4, W=128, H=128, K=5, L=20, gamma=1.0, loss=4, n_blobs=(2, 5)),  # batched shape, short L
    dict(P=3, W=72, H=40, K=3, L=10, gamma=2.0, loss=1),             # ragged, non-square
    dict(P=2, W=24, H=20, D=12, K=2, L=6, gamma=2.0, loss=2),        # 3-D
])
def test_evaluate_vs_oracle(oracle, case, precision):
    case = dict(case)
    D = case.pop("D", 1)
    cfg, obs, x = _problem(D=D, **case)
    W, H, P, K, L = cfg["W"], cfg["H"], cfg["P"], cfg["K"], cfg["L"]
    f_ref, g_ref = oracle.evaluate_both(W, H, D, cfg["gamma"], P, K, L, cfg["loss"], cfg["scale_dic"],
                                        x, obs)
    reg = _regression(W, H, D, cfg["gamma"], P, K, L, cfg["loss"], cfg["scale_dic"], obs, precision)
    fv, g = reg.evaluate_both(x)
    tol = TOL[precision]
    assert abs(fv - f_ref) <= tol * abs(f_ref)
    check_gradient(oracle, g, g_ref, W, H, D, cfg["gamma"], P, K, L, cfg["loss"], cfg["scale_dic"],
                   x, obs, tol, tol)


def test_batch_invariance_and_determinism():
    """Each histogram's outputs are the same alone and inside the batch; two
    runs are bit-identical (no atomics in any reduction)."""
    cfg, obs, x = _problem(P=6, W=48, H=40, K=3, L=12, gamma=2.0, loss=2)
    W, H, P, K, L = cfg["W"], cfg["H"], cfg["P"], cfg["K"], cfg["L"]
    from wassersteindictionarylearning_b200.synthetic import init_atoms, init_weights
    atoms = init_atoms(K, W * H, seed=7)
    w = init_weights(P, K, seed=8)
    reg = _regression(W, H, 1, cfg["gamma"], P, K, L, cfg["loss"], 1.0, obs, "fp32")
    la, dic, bary, loss = reg.compute_gradient_both(atoms, w)
    la2, dic2, bary2, loss2 = reg.compute_gradient_both(atoms, w)
    assert np.array_equal(la, la2) and np.array_equal(dic, dic2) and np.array_equal(bary, bary2)
    for p in (0, 3, 5):
        one = _regression(W, H, 1, cfg["gamma"], 1, K, L, cfg["loss"], 1.0, obs[p], "fp32")
        la1, dic1, bary1, loss1 = one.compute_gradient_both(atoms, w[p])
        assert np.array_equal(bary1, bary[p * W * H:(p + 1) * W * H])
        assert np.array_equal(la1, la[p * K:(p + 1) * K])
        assert loss1[0] == loss[p]


def test_edge_cases():
    from wassersteindictionarylearning_b200 import WdlError, _lib
    import ctypes as C
    L = _lib.lib()
    h = C.c_void_p()
    assert L.wdl_create(C.byref(h), -1, 0, 8, 1, 1.0, 0, 0) == -1      # empty grid
    assert L.wdl_create(C.byref(h), -1, 8, 8, 1, -1.0, 0, 0) == -1     # bad gamma
    assert L.wdl_create(C.byref(h), -1, 8, 8, 2, 1.0, 0, 1) == -4      # 3-D log domain
    k = kern(2.0, 1, 1)                                                # 1x1 grid
    assert np.allclose(k.convolve(np.array([3.0])), [3.0])
    k = kern(2.0, 8, 8)
    assert k.convolve(np.zeros(0), 0).size == 0                        # zero images
    with pytest.raises(WdlError):
        _regression(8, 8, 1, 2.0, 1, 2, 3, 7, 1.0, np.ones(64) / 64, "fp32").compute_gradient_both(
            np.ones(128), np.ones(2))                                  # unknown loss


# ---- tensor-core forms --------------------------------------------------------------
# Operator tolerance against FP64: TF32 (10-bit mantissa) ~1e-3, split BF16
# (hi+lo, three products, FP32 accumulate) ~1e-5.  Whole-path targets against
# FP64: barycenter <= 1e-4 and gradients <= 1e-3 (split BF16).
TC_OP_TOL = {"tf32": 3e-3, "split_bf16": 2e-5}


@pytest.mark.parametrize("precision", ["split_bf16", "tf32"])
@pytest.mark.parametrize("name,f", [g for g in golden("conv_*") if int(g[1]["D"]) == 1])
def test_convolve_tensor_core(name, f, precision):
    k = kern(float(f["gamma"]), int(f["W"]), int(f["H"]), 1, precision)
    out = k.convolve(f["u"], int(f["nv"]))
    assert rel(out, f["out"]) < TC_OP_TOL[precision]


@pytest.mark.parametrize("shape", [(128, 128), (64, 64), (100, 72), (17, 128), (128, 33)])
def test_convolve_tensor_core_shapes(oracle, shape):
    W, H = shape
    rng = np.random.default_rng(W * 1000 + H)
    u = rng.random(3 * W * H)
    ref = oracle.convolve(W, H, 1, 1.5, u, 3)
    for precision, tol in TC_OP_TOL.items():
        out = kern(1.5, W, H, 1, precision).convolve(u, 3)
        assert rel(out, ref) < tol, precision


@pytest.mark.parametrize("case", [
    dict(P=16, W=64, H=64, K=4, L=25, gamma=2.0, loss=2),
    dict(P=4, W=128, H=128, K=5, L=30, gamma=1.0, loss=4, n_blobs=(2, 5)),
])
def test_split_bf16_path_vs_oracle(oracle, case):
    case = dict(case)
    cfg, obs, x = _problem(**case)
    W, H, P, K, L = cfg["W"], cfg["H"], cfg["P"], cfg["K"], cfg["L"]
    f_ref, g_ref, bary_ref = oracle.evaluate_both(W, H, 1, cfg["gamma"], P, K, L, cfg["loss"],
                                                  cfg["scale_dic"], x, obs, want_bary=True)
    reg = _regression(W, H, 1, cfg["gamma"], P, K, L, cfg["loss"], cfg["scale_dic"], obs,
                      "split_bf16")
    fv, g = reg.evaluate_both(x)
    assert rel(reg.last_barycenters, bary_ref) < 1e-4
    assert abs(fv - f_ref) <= 1e-4 * abs(f_ref)
    check_gradient(oracle, g, g_ref, W, H, 1, cfg["gamma"], P, K, L, cfg["loss"], cfg["scale_dic"],
                   x, obs, 1e-3, 1e-3)


@pytest.mark.parametrize("precision", ["split_bf16", "tf32"])
def test_fused_gradient_both_vs_oracle(oracle, precision):
    """Raw resultLa / resultDic / barycenters / losses of the persistent fused
    kernel against the FP64 oracle, histogram by histogram."""
    cfg, obs, x = _problem(P=5, W=48, H=40, K=3, L=15, gamma=1.5, loss=2)
    W, H, P, K, L = cfg["W"], cfg["H"], cfg["P"], cfg["K"], cfg["L"]
    from wassersteindictionarylearning_b200.synthetic import init_atoms, init_weights
    atoms = init_atoms(K, W * H, seed=3)
    w = init_weights(P, K, seed=4)
    reg = _regression(W, H, 1, cfg["gamma"], P, K, L, 2, 1.0, obs, precision)
    la, dic, bary, loss = reg.compute_gradient_both(atoms, w)
    tol_b, tol_g = (1e-4, 1e-3) if precision == "split_bf16" else (3e-3, 2e-2)
    dic_ref = np.zeros(K * W * H)
    for p in range(P):
        la_r, dic_r, bary_r = oracle.gradient_both(W, H, 1, cfg["gamma"], K, L, 2, atoms, w[p], obs[p])
        f_r, _ = oracle.loss(2, W, H, 1, cfg["gamma"], bary_r, obs[p])
        scale = oracle.gradient_both_scale(W, H, 1, cfg["gamma"], K, L, 2, atoms, w[p], obs[p])
        assert rel(bary[p * W * H:(p + 1) * W * H], bary_r) < tol_b
        assert abs(loss[p] - f_r) <= tol_b * abs(f_r)
        assert rel_scaled(la[p * K:(p + 1) * K], la_r, scale) < tol_g
        dic_ref += dic_r
    assert rel(dic, dic_ref) < tol_g


def test_fused_barycenter_and_warm_restart(oracle):
    from wassersteindictionarylearning_b200 import Problem, WassersteinBarycenter
    (_, f), = golden("bary_16x16x1_K3_L20_ker")
    k = kern(float(f["gamma"]), 16, 16, 1, "split_bf16")
    prob = Problem(f["atoms"], np.zeros(256), k, f["lambdas"], 1)
    b = WassersteinBarycenter(prob, int(f["L"])).compute_barycenter()
    assert rel(b, f["bary"]) < 1e-4
    # several weight vectors at once (the serving batch form)
    from wassersteindictionarylearning_b200.synthetic import init_weights
    ws = init_weights(7, 3, seed=9)
    bs = WassersteinBarycenter(prob, int(f["L"])).compute_barycenter(ws)
    for i in range(7):
        ref = oracle.barycenter(16, 16, 1, float(f["gamma"]), 3, int(f["L"]), f["atoms"], ws[i])
        assert rel(bs[i], ref) < 1e-4
    (_, f), = golden("warm_*")
    W, H, P, K, L = (int(f[k]) for k in ("W", "H", "P", "K", "L"))
    reg = _regression(W, H, 1, float(f["gamma"]), P, K, L, int(f["loss"]), float(f["scale_dic"]),
                      f["obs"], "split_bf16")
    reg.warmRestart = True
    reg.b_storage = f["b_storage"].copy()
    fv, g = reg.evaluate_both(f["x"])
    assert abs(fv - float(f["f"])) <= 1e-4 * abs(float(f["f"]))
    assert rel(reg.b_temp, f["b_last"]) < 1e-4
    assert rel(g[P * K:], f["g"][P * K:]) < 1e-3


def test_fused_wasserstein_loss_falls_back_to_operator_path(oracle):
    """Loss type 3 (nested Sinkhorn) runs through the unfused tensor-core
    operator path; results still match the oracle."""
    cfg, obs, x = _problem(P=2, W=16, H=16, K=2, L=5, gamma=2.0, loss=3)
    W, H, P, K, L = cfg["W"], cfg["H"], cfg["P"], cfg["K"], cfg["L"]
    f_ref, g_ref = oracle.evaluate_both(W, H, 1, 2.0, P, K, L, 3, cfg["scale_dic"], x, obs)
    reg = _regression(W, H, 1, 2.0, P, K, L, 3, cfg["scale_dic"], obs, "split_bf16")
    fv, g = reg.evaluate_both(x)
    assert abs(fv - f_ref) <= 1e-3 * abs(f_ref)
    assert rel(g[P * K:], g_ref[P * K:]) < 1e-2
