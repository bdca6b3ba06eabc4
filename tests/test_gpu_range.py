"""GPU: kernel-domain scalings beyond the FP32 range.

With a narrow kernel (gamma 2 px^2) and atoms with empty regions, the
kernel-domain scalings pass 1e60 within 50 iterations: inside the range of
FP64 (the reference's arithmetic), beyond that of FP32.  The FP32 forms
(SIMT FP32, TF32, split BF16; fused kernel up to 128, axis passes above) must
not return finite values computed from saturated scalings: the affected
histograms' barycenters, losses and weight gradients come back NaN, where the
FP64 path returns finite values."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("W,precision", [(64, "split_bf16"), (64, "tf32"), (64, "fp32"),
                                         (160, "split_bf16")])
def test_out_of_range_scalings_come_back_nan(W, precision):
    from wassersteindictionarylearning_b200 import CudaGaussian2DKernel
    from wassersteindictionarylearning_b200._lib import check, dptr, lib
    from wassersteindictionarylearning_b200.synthetic import blob_histograms
    K, L, P = 5, 50, 2
    N = W * W
    atoms = np.ascontiguousarray(blob_histograms(K, W, W, 1, n_blobs=(1, 3), seed=100))
    obs = np.ascontiguousarray(blob_histograms(P, W, W, 1, n_blobs=(1, 3), seed=101))
    w = np.full((P, K), 1.0 / K)
    out = {}
    for prec in (precision, "fp64"):
        k = CudaGaussian2DKernel(2.0, W, W, precision=prec)
        bary = np.empty(P * N)
        check(lib().wdl_barycenter(k.ctx, P, K, L, dptr(atoms), dptr(w), dptr(bary)), k.ctx)
        la, dic, loss = np.empty(P * K), np.empty(K * N), np.empty(P)
        check(lib().wdl_gradient_both(k.ctx, P, K, L, 2, dptr(atoms), dptr(w), dptr(obs), None,
                                      dptr(la), dptr(dic), None, dptr(loss), None), k.ctx)
        out[prec] = (bary, la, loss)
        k.close()
    for a in out["fp64"]:
        assert np.all(np.isfinite(a))
    # the forward pass of every histogram meets the overflow (it depends on the
    # atoms and the uniform weights only)
    for a in out[precision]:
        assert np.all(np.isnan(a)), precision
