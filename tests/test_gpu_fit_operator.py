"""GPU: wdl_fit_weights_operator, the weight fits of regress_both with the
atoms held fixed (cpp/inverseWasserstein.h:362-423; liblbfgs,
cpp/lbfgs/lbfgs.c:256-654, :772-867) with the L-BFGS on the device around the
context's own evaluation path.  On an FP64 context the device optimisation
must take the decisions the host L-BFGS (lbfgs.lbfgs_steps) takes around
wdl_gradient_both on the same context: same status, same number of
evaluations, the same weights and loss to the FP64 rounding of the steps."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _problem(W, H, D, K, P, seed):
    from wassersteindictionarylearning_b200.synthetic import blob_histograms
    N = W * H * D
    atoms = blob_histograms(K, W, H, D, seed=seed).reshape(K, N) + 1.0 / N
    atoms /= atoms.sum(axis=1, keepdims=True)
    obs = blob_histograms(P, W, H, D, seed=seed + 1).reshape(P, N)
    return np.ascontiguousarray(atoms.reshape(-1)), np.ascontiguousarray(obs.reshape(-1))


def _host_fit(ctx, K, L, atoms, obs_p, iters, eps):
    from wassersteindictionarylearning_b200 import lbfgs as lb
    from wassersteindictionarylearning_b200._lib import check, dptr, lib
    gen = lb.lbfgs_steps(np.zeros(K), lb.LbfgsParam(max_iterations=iters, epsilon=eps))
    x = next(gen)
    evals = 0
    seen = {}
    while True:
        w = np.exp(x - x.max())
        w /= w.sum()
        la, loss = np.empty(K), np.empty(1)
        check(lib().wdl_gradient_both(ctx, 1, K, L, 2, dptr(atoms), dptr(w), dptr(obs_p), None, dptr(la),
                                      None, None, dptr(loss), None), ctx)
        evals += 1
        seen[x.tobytes()] = float(loss[0])
        try:
            x = gen.send((float(loss[0]), (la - np.dot(w, la)) * w))
        except StopIteration as e:
            st, xr, fx = e.value
            wr = np.exp(xr - xr.max())
            return wr / wr.sum(), seen.get(xr.tobytes(), fx), st, evals


@pytest.mark.parametrize("W,H,D", [(20, 16, 1), (8, 6, 5)])
def test_device_fit_matches_host_fit(W, H, D):
    from wassersteindictionarylearning_b200 import CudaGaussian2DKernel, CudaGaussian3DKernel
    from wassersteindictionarylearning_b200._lib import check, dptr, lib
    K, L, P, iters, eps = 3, 8, 3, 10, 1e-8
    atoms, obs = _problem(W, H, D, K, P, seed=70 + D)
    kern = (CudaGaussian2DKernel(1.5, W, H, precision="fp64") if D == 1
            else CudaGaussian3DKernel(1.5, W, H, D, precision="fp64"))
    w = np.empty(P * K)
    f = np.empty(P)
    st = np.zeros(P, dtype=np.int32)
    ev = np.zeros(P, dtype=np.int32)
    ip = C.POINTER(C.c_int)
    check(lib().wdl_fit_weights_operator(kern.ctx, P, K, L, 2, dptr(atoms), dptr(obs), None, iters, eps,
                                         dptr(w), dptr(f), st.ctypes.data_as(ip), ev.ctypes.data_as(ip)),
          kern.ctx)
    N = W * H * D
    for p in range(P):
        wh, fh, sth, evh = _host_fit(kern.ctx, K, L, atoms, np.ascontiguousarray(obs[p * N:(p + 1) * N]),
                                     iters, eps)
        assert st[p] == sth and ev[p] == evh, (p, st[p], sth, ev[p], evh)
        assert abs(f[p] - fh) <= 1e-10 * abs(fh)
        assert np.max(np.abs(w[p * K:(p + 1) * K] - wh)) < 1e-8
        assert abs(w[p * K:(p + 1) * K].sum() - 1) < 1e-12
    kern.close()


def test_device_fit_refuses_the_fused_context():
    from wassersteindictionarylearning_b200 import CudaGaussian2DKernel
    from wassersteindictionarylearning_b200._lib import dptr, lib
    K, P = 2, 1
    atoms, obs = _problem(16, 16, 1, K, P, seed=3)
    kern = CudaGaussian2DKernel(1.5, 16, 16, precision="split_bf16")
    w, f = np.empty(P * K), np.empty(P)
    st, ev = np.zeros(P, dtype=np.int32), np.zeros(P, dtype=np.int32)
    ip = C.POINTER(C.c_int)
    rc = lib().wdl_fit_weights_operator(kern.ctx, P, K, 5, 2, dptr(atoms), dptr(obs), None, 3, 1e-8,
                                        dptr(w), dptr(f), st.ctypes.data_as(ip), ev.ctypes.data_as(ip))
    assert rc == -4  # WDL_ERR_UNSUPPORTED
    kern.close()
