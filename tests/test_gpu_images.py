"""GPU, end to end from image files: images -> histograms (histio, the
reference's conversions) -> dictionary learning with regress_both on the CUDA
KernelType -> atoms and reconstructions written back as images."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_dictionary_learning_from_image_files(tmp_path):
    from wassersteindictionarylearning_b200 import (CudaGaussian2DKernel, Problem,
                                                    WassersteinRegression)
    from wassersteindictionarylearning_b200 import histio as hio
    from wassersteindictionarylearning_b200.synthetic import blob_histograms, init_atoms, init_weights
    W, H, P, K, L = 40, 32, 4, 2, 20
    imgs = blob_histograms(P, W, H, seed=21)
    names = []
    for p in range(P):  # grey images as the reference's inputs would be
        g = imgs[p].reshape(H, W)
        path = str(tmp_path / f"in{p}{'.png' if p % 2 else '.pgm'}")
        hio.write_image(path, np.clip(g / g.max() * 255.0, 0, 255).astype(np.uint8))
        names.append(path)
    loaded = [hio.load_img_to_pdf(n) for n in names]
    assert all((w, h) == (W, H) for _, w, h, _ in loaded)
    obs = np.stack([pdf for pdf, *_ in loaded])
    k = CudaGaussian2DKernel(4.0, W, H, precision="split_bf16")
    atoms = init_atoms(K, W * H, seed=22)
    weights = init_weights(P, K, seed=23)
    sd = (W * H / P) / 100.0
    reg = WassersteinRegression(Problem(atoms, obs, k, None, P), L, 2, sd)
    reg.wrTotalIteration = 6  # regress_both runs this many L-BFGS iterations
    x0 = np.concatenate([weights.reshape(-1), atoms.reshape(-1)])
    f0, _ = reg.evaluate_both(np.concatenate([np.log(weights.reshape(-1)) * sd, np.log(atoms.reshape(-1))]))
    sol = x0.copy()
    reg.regress_both(sol)
    w_fit, a_fit = sol[:P * K].reshape(P, K), sol[P * K:].reshape(K, W * H)
    f1, _ = reg.evaluate_both(np.concatenate([np.log(w_fit.reshape(-1)) * sd, np.log(a_fit.reshape(-1))]))
    assert f1 < f0
    assert np.allclose(w_fit.sum(axis=1), 1) and np.allclose(a_fit.sum(axis=1), 1)
    out = str(tmp_path / "out")
    os.makedirs(out)
    assert hio.ExportHistogramToImage(W, H, out).exportHistogramsBatch(list(a_fit), ["atom0", "atom1"]) == 0
    scal = [s for *_, s in loaded]
    recon = reg.last_barycenters.reshape(P, -1)
    ex = hio.ExportHistogramToImageWithScaling(W, H, scal, out)
    assert ex.exportHistogramsBatch(list(recon), [f"rec{p}" for p in range(P)]) == 0
    back = hio.read_image(os.path.join(out, "atom0.png"))
    # the reference's exporters write the grey plane in three channels
    assert back.shape == (H, W, 3) and back.max() > 0 and (back == back[:, :, :1]).all()
    k.close()
