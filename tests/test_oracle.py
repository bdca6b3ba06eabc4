"""CPU tests: the oracle pinned to the reference's own outputs.

The reference ships no tests or fixtures; its outputs on seeded inputs were
recorded by tests/golden/make_golden.py into tests/golden/*.npz.  These tests
check the C restatement of the oracle against them (FP64, to rounding), and the
reference build itself when its sources are present.
"""
import numpy as np
import pytest

from conftest import golden, rel
from oracle import oracle as orc

TOL = 1e-11  # FP64 restatement vs reference: summation order is the same


@pytest.mark.parametrize("name,f", golden("conv_*"))
def test_conv_golden(oracle, name, f):
    out = oracle.convolve(int(f["W"]), int(f["H"]), int(f["D"]), float(f["gamma"]), f["u"], int(f["nv"]))
    assert rel(out, f["out"]) < 1e-14


@pytest.mark.parametrize("name,f", golden("logconv_*"))
def test_logconv_golden(oracle, name, f):
    W, H, g, nv = int(f["W"]), int(f["H"]), float(f["gamma"]), int(f["nv"])
    assert rel(oracle.log_convolve(W, H, g, f["u"], nv), f["out"]) < 1e-14
    out, signs = oracle.log_convolve_signed(W, H, g, f["u"], f["signs_in"], nv)
    assert rel(out, f["out_signed"]) < 1e-14
    assert np.array_equal(signs, f["signs_out"])


def test_loss_golden(oracle):
    (_, f), = golden("loss_10x9")
    for lt in (1, 2, 3, 4):
        val, gr = oracle.loss(lt, 10, 9, 1, float(f["gamma"]), f["v1"], f["v2"])
        assert abs(val - float(f[f"f{lt}"])) <= 1e-12 * abs(float(f[f"f{lt}"]))
        assert rel(gr, f[f"g{lt}"]) < 1e-12


@pytest.mark.parametrize("name,f", golden("grad_*"))
def test_gradient_both_golden(oracle, name, f):
    la, dic, bary = oracle.gradient_both(int(f["W"]), int(f["H"]), int(f["D"]), float(f["gamma"]),
                                         int(f["K"]), int(f["L"]), int(f["loss"]), f["atoms"],
                                         f["lambdas"], f["obs"])
    assert rel(bary, f["bary"]) < TOL
    assert rel(dic, f["resultDic"]) < TOL
    assert rel(la, f["resultLa"]) < 1e-10


@pytest.mark.parametrize("name,f", golden("gradlog_*"))
def test_gradient_both_log_golden(oracle, name, f):
    la, dic, bary = oracle.gradient_both_log(int(f["W"]), int(f["H"]), float(f["gamma"]),
                                             int(f["K"]), int(f["L"]), int(f["loss"]), f["atoms"],
                                             f["lambdas"], f["obs"])
    assert rel(bary, f["bary"]) < TOL
    assert rel(dic, f["resultDic"]) < 1e-10
    assert rel(la, f["resultLa"]) < 1e-10


@pytest.mark.parametrize("name,f", golden("bary_*"))
def test_barycenter_golden(oracle, name, f):
    b = oracle.barycenter(int(f["W"]), int(f["H"]), int(f["D"]), float(f["gamma"]), int(f["K"]),
                          int(f["L"]), f["atoms"], f["lambdas"], log_domain=bool(f["log"]))
    assert rel(b, f["bary"]) < TOL


@pytest.mark.parametrize("name,f", golden("eval_*"))
def test_evaluate_both_golden(oracle, name, f):
    fv, g = oracle.evaluate_both(int(f["W"]), int(f["H"]), int(f["D"]), float(f["gamma"]),
                                 int(f["P"]), int(f["K"]), int(f["L"]), int(f["loss"]),
                                 float(f["scale_dic"]), f["x"], f["obs"], log_domain=bool(f["log"]))
    assert abs(fv - float(f["f"])) <= 1e-12 * abs(float(f["f"]))
    assert rel(g, f["g"]) < 1e-10


def test_warm_restart_golden(oracle):
    (_, f), = golden("warm_*")
    fv, g, bl = oracle.evaluate_both(int(f["W"]), int(f["H"]), 1, float(f["gamma"]), int(f["P"]),
                                     int(f["K"]), int(f["L"]), int(f["loss"]), float(f["scale_dic"]),
                                     f["x"], f["obs"], b_storage=f["b_storage"], want_b_last=True)
    assert abs(fv - float(f["f"])) <= 1e-12 * abs(float(f["f"]))
    assert rel(g, f["g"]) < 1e-10
    assert rel(bl, f["b_last"]) < TOL


@pytest.mark.skipif(not orc.ref_available(), reason="reference build (oracle/_ref) absent")
def test_reference_build_matches_golden():
    R = orc.RefLib()
    (_, f), = golden("eval_P3_16x16x1_K3_L10_loss2_ker")
    fv, g = R.evaluate_both(16, 16, 1, float(f["gamma"]), 3, 3, 10, 2, float(f["scale_dic"]), f["x"], f["obs"])
    assert fv == float(f["f"])
    assert rel(g, f["g"]) < 1e-15


@pytest.mark.skipif(not orc.ref_available(), reason="reference build (oracle/_ref) absent")
def test_reference_sse_kernel_agrees():
    R = orc.RefLib()
    rng = np.random.default_rng(3)
    u = rng.random(2 * 32 * 24)
    a = R.convolve(32, 24, 1, 2.0, u, 2)
    b = R.convolve(32, 24, 1, 2.0, u, 2, sse=True)
    assert rel(a, b) < 1e-13
