"""GPU: every output of evaluate_both against the FP64 oracle, for every
precision, on the batched 128x128 configuration (P reduced to 4 histograms,
full L = 100, gamma 1, KL loss, 2-5 blob histograms, uniform+noise atoms).

Asserts the stated bounds and prints the measured errors (run with -s):
barycenters and the atom gradient normwise relative; the loss relative; the
weight gradient against its condition scale (the mass of the terms summed
into it, oracle.weight_gradient_scale)."""
import json

import numpy as np
import pytest

from conftest import rel, rel_scaled

pytestmark = pytest.mark.gpu

BOUNDS = {  # precision: (barycenter, loss, atom gradient, weight gradient)
    "fp64": (1e-10, 1e-10, 1e-10, 1e-10),
    "fp32": (1e-5, 1e-5, 1e-5, 1e-5),
    "tf32": (3e-3, 3e-3, 2e-2, 2e-2),
    "split_bf16": (1e-4, 1e-4, 1e-3, 1e-3),
}


def test_precision_report(oracle):
    from wassersteindictionarylearning_b200 import (CudaGaussian2DKernel, Problem,
                                                    WassersteinRegression)
    from wassersteindictionarylearning_b200.synthetic import make_problem, to_variables
    P, W, H, K, L, gamma, loss = 4, 128, 128, 5, 100, 1.0, 4
    cfg, obs, atoms, w = make_problem(None, seed=0, P=P, W=W, H=H, K=K, L=L, gamma=gamma,
                                      loss=loss, n_blobs=(2, 5))
    sd = cfg["scale_dic"]
    x = to_variables(w, atoms, sd)
    f_ref, g_ref, bary_ref = oracle.evaluate_both(W, H, 1, gamma, P, K, L, loss, sd, x, obs,
                                                  want_bary=True)
    scale = oracle.weight_gradient_scale(W, H, 1, gamma, P, K, L, loss, sd, x, obs)
    PK = P * K
    report = {}
    for prec, (tb, tf, ta, tw) in BOUNDS.items():
        k = CudaGaussian2DKernel(gamma, W, H, precision=prec)
        reg = WassersteinRegression(Problem(np.ones((K, W * H)), obs, k, None, P), L, loss, sd)
        fv, g = reg.evaluate_both(x)
        e = dict(barycenter=rel(reg.last_barycenters, bary_ref), loss=abs(fv - f_ref) / abs(f_ref),
                 atom_gradient=rel(g[PK:], g_ref[PK:]),
                 weight_gradient=rel_scaled(g[:PK], g_ref[:PK], scale))
        report[prec] = e
        k.close()
        assert e["barycenter"] < tb and e["loss"] < tf, (prec, e)
        assert e["atom_gradient"] < ta and e["weight_gradient"] < tw, (prec, e)
    print("\nPRECISION_REPORT " + json.dumps(report))
