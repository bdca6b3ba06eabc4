"""GPU: the weight gradient alone (result_dic = NULL).

Fitting weights onto a fixed dictionary needs no atom gradient; passing NULL
for it skips the dictionary recursion in the kernel domain.  The weight
recursion does not read the dictionary one, so the weight gradients, losses and
barycenters must equal those of the full call: bitwise on the CUDA-core forms
(the operator treats every image alike, alone or in the [dictionary | weights]
pair), within the run-to-run rounding of the fused tensor-core kernel's float
accumulations otherwise.  The log domain computes both recursions either way."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision,W,exact", [("fp64", 40, True), ("fp32", 40, True),
                                               ("fp64", 24, True), ("split_bf16", 48, False),
                                               ("split_bf16", 136, True)])
def test_weights_only_matches_full_call(precision, W, exact):
    from wassersteindictionarylearning_b200 import CudaGaussian2DKernel
    from wassersteindictionarylearning_b200._lib import check, dptr, lib
    from wassersteindictionarylearning_b200.synthetic import blob_histograms, init_weights
    H, K, L, P = W - 4, 3, 9, 2
    N = W * H
    atoms = np.ascontiguousarray(blob_histograms(K, W, H, seed=3) + 1.0 / N)
    obs = np.ascontiguousarray(blob_histograms(P, W, H, seed=4))
    w = np.ascontiguousarray(init_weights(P, K, seed=5))
    k = CudaGaussian2DKernel(4.0, W, H, precision=precision)
    out = []
    for want_dic in (True, False, True, False):
        la, loss, bary = np.empty(P * K), np.empty(P), np.empty(P * N)
        dic = np.empty(K * N) if want_dic else None
        check(lib().wdl_gradient_both(k.ctx, P, K, L, 2, dptr(atoms), dptr(w), dptr(obs), None,
                                      dptr(la), dptr(dic) if want_dic else None, dptr(bary),
                                      dptr(loss), None), k.ctx)
        out.append((la, loss, bary))
    k.close()
    full, alone = out[0], out[1]
    for a, b in zip(full, alone):
        assert np.all(np.isfinite(b))
        if exact:
            assert np.array_equal(a, b)
        else:
            assert np.max(np.abs(a - b)) <= 1e-5 * np.max(np.abs(a))
    # repeated calls (graph-replayed on the CUDA-core forms) give the same again
    for a, b in zip(out[1], out[3]):
        assert np.array_equal(a, b) or not exact
