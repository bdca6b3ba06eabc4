"""CPU tests of the host side: the C ABI library loads and exports every symbol
that include/wdl.h declares (no compute call without a GPU), the library fails
loudly without a device, the synthetic generator, and the host L-BFGS driving
the oracle's objective against the reference's own regress_both run."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import ROOT, golden, rel


def header_symbols():
    txt = open(os.path.join(ROOT, "include", "wdl.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(wdl_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    from wassersteindictionarylearning_b200 import _lib
    if not os.path.exists(_lib.LIB_PATH):
        _lib.build()
    L = C.CDLL(_lib.LIB_PATH)
    syms = header_symbols()
    assert len(syms) >= 19
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, missing
    # the ctypes table covers the header too
    assert set(_lib.SIGNATURES) == set(syms)


def test_no_device_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from wassersteindictionarylearning_b200 import _lib
    h = C.c_void_p()
    rc = _lib.lib().wdl_create(C.byref(h), -1, 8, 8, 1, 1.0, 0, 0)
    assert rc == -8  # WDL_ERR_NO_DEVICE: no silent CPU fallback
    assert b"device" in _lib.lib().wdl_last_error(None)
    assert _lib.lib().wdl_strerror(-8) == b"no usable sm_100 CUDA device"


def test_kernel_object_raises_without_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from wassersteindictionarylearning_b200 import CudaGaussian2DKernel, WdlError
    with pytest.raises(WdlError):
        CudaGaussian2DKernel(2.0, 16, 16)


def test_synthetic_histograms():
    from wassersteindictionarylearning_b200.synthetic import blob_histograms, init_atoms, init_weights
    h = blob_histograms(4, 32, 24, seed=0)
    assert h.shape == (4, 32 * 24)
    assert np.allclose(h.sum(axis=1), 1.0)
    assert (h > 0).all()
    assert np.array_equal(h, blob_histograms(4, 32, 24, seed=0))
    h3 = blob_histograms(2, 8, 6, 5, seed=1)
    assert h3.shape == (2, 240) and np.allclose(h3.sum(axis=1), 1.0)
    a = init_atoms(3, 100)
    assert np.allclose(a.sum(axis=1), 1.0)
    w = init_weights(5, 3)
    assert np.allclose(w.sum(axis=1), 1.0)


def test_lbfgs_matches_reference_regress_both(oracle):
    """Host L-BFGS over the oracle objective reproduces the reference's
    regress_both (liblbfgs, strong-Wolfe backtracking) for a few iterations."""
    from wassersteindictionarylearning_b200 import lbfgs as lb
    (_, f), = golden("regress_*")
    P, W, H, K, L = int(f["P"]), int(f["W"]), int(f["H"]), int(f["K"]), int(f["L"])
    sd, lt, g = float(f["scale_dic"]), int(f["loss"]), float(f["gamma"])
    N = W * H
    sol0 = f["solution0"]
    x0 = np.concatenate([np.log(sol0[:P * K]) * sd, np.log(sol0[P * K:])])

    def ev(x, step):
        return oracle.evaluate_both(W, H, 1, g, P, K, L, lt, sd, x, f["obs"])

    p = lb.LbfgsParam(max_iterations=int(f["iters"]))
    ret, x, _ = lb.lbfgs(x0, ev, None, p)
    assert ret == lb.LBFGSERR_MAXIMUMITERATION
    w = np.exp(x[:P * K] / sd).reshape(P, K)
    w /= w.sum(axis=1, keepdims=True)
    a = np.exp(x[P * K:]).reshape(K, N)
    a /= a.sum(axis=1, keepdims=True)
    sol = np.concatenate([w.reshape(-1), a.reshape(-1)])
    assert rel(sol, f["solution"]) < 1e-8


def test_lbfgs_quadratic():
    from wassersteindictionarylearning_b200 import lbfgs as lb
    A = np.diag(np.arange(1.0, 11.0))
    b = np.ones(10)

    def ev(x, step):
        return 0.5 * x @ A @ x - b @ x, A @ x - b

    ret, x, fx = lb.lbfgs(np.zeros(10), ev, None, lb.LbfgsParam(epsilon=1e-6, max_iterations=100))
    assert ret == lb.LBFGS_SUCCESS
    assert np.allclose(x, 1.0 / np.arange(1.0, 11.0), atol=1e-5)


def test_lbfgs_cancel_on_nan():
    from wassersteindictionarylearning_b200 import lbfgs as lb

    def ev(x, step):
        return float("nan") if step > 0 else 1.0, np.ones_like(x)

    def prog(x, g, fx, xn, gn, step, k, ls):
        return lb.LBFGSERR_CANCELED if np.isnan(fx) else 0

    ret, _, _ = lb.lbfgs(np.zeros(3), ev, prog, lb.LbfgsParam(max_iterations=5))
    # NaN fails the sufficient-decrease test until the trial budget runs out
    assert ret in (lb.LBFGSERR_CANCELED, lb.LBFGSERR_MAXIMUMLINESEARCH)


def test_resumable_lbfgs_matches_blocking_form():
    from wassersteindictionarylearning_b200 import lbfgs as lb
    A = np.diag(np.linspace(1.0, 30.0, 12))
    b = np.linspace(-1, 1, 12)

    def ev(x, step=0.0):
        return 0.5 * x @ A @ x - b @ x, A @ x - b

    p = lb.LbfgsParam(max_iterations=15)
    r1, x1, f1 = lb.lbfgs(np.zeros(12), ev, None, p)
    gen = lb.lbfgs_steps(np.zeros(12), p)
    x = next(gen)
    try:
        while True:
            x = gen.send(ev(x))
    except StopIteration as e:
        r2, x2, f2 = e.value
    assert r1 == r2 and np.array_equal(x1, x2) and f1 == f2


def test_host_lbfgs_reproduces_reference_regress_both(oracle):
    """The host L-BFGS (one copy of liblbfgs' algorithm, lbfgs.py) driven by the
    oracle's evaluate_both lands where the reference's regress_both does after
    four iterations (golden regress_*, cpp/inverseWasserstein.h:362-423)."""
    from conftest import golden, rel
    from wassersteindictionarylearning_b200 import lbfgs as lb
    (_, f), = golden("regress_*")
    W, H, P, K, L = (int(f[k]) for k in ("W", "H", "P", "K", "L"))
    sd, g, lt = float(f["scale_dic"]), float(f["gamma"]), int(f["loss"])
    sol0 = f["solution0"]
    x0 = np.concatenate([np.log(sol0[: P * K]) * sd, np.log(sol0[P * K:])])

    def ev(x, step):
        return oracle.evaluate_both(W, H, 1, g, P, K, L, lt, sd, x, f["obs"])

    ret, x, _ = lb.lbfgs(x0, ev, None, lb.LbfgsParam(max_iterations=int(f["iters"])))
    w = np.exp(x[: P * K] / sd).reshape(P, K)
    w /= w.sum(axis=1, keepdims=True)
    a = np.exp(x[P * K:]).reshape(K, -1)
    a /= a.sum(axis=1, keepdims=True)
    assert rel(np.concatenate([w.reshape(-1), a.reshape(-1)]), f["solution"]) < 1e-8
