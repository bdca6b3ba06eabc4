"""Generate the golden fixtures in this folder from the reference's own code.

Runs the UNMODIFIED reference (compiled by oracle/Makefile into oracle/_ref from
the reference sources) on small seeded inputs and stores inputs and outputs as
compressed .npz files.  The reference ships no tests or fixtures of its own, so
these runs are what pins the oracle and the CUDA path.

    python tests/golden/make_golden.py      # needs oracle/_ref (reference sources present)
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.oracle import RefLib  # noqa: E402
from wassersteindictionarylearning_b200.synthetic import (blob_histograms, init_atoms,  # noqa: E402
                                                          init_weights, scale_dictionary,
                                                          to_variables)


def save(name, **arrays):
    path = os.path.join(HERE, name + ".npz")
    np.savez_compressed(path, **{k: np.asarray(v) for k, v in arrays.items()})
    print("wrote", path, os.path.getsize(path), "bytes")


def main():
    R = RefLib()
    rng = np.random.Generator(np.random.PCG64(1234))

    # Operator fixtures (cpp/kernels.h): non-square and 3-D sizes, several images.
    for (W, H, D, g, nv) in [(16, 12, 1, 2.0, 3), (33, 20, 1, 1.0, 2), (6, 5, 4, 2.0, 2),
                             (48, 48, 1, 0.5, 1)]:
        u = rng.random(nv * W * H * D)
        save(f"conv_{W}x{H}x{D}_g{g}", W=W, H=H, D=D, gamma=g, nv=nv, u=u,
             out=R.convolve(W, H, D, g, u, nv))
    for (W, H, g, nv) in [(12, 9, 0.5, 2), (20, 16, 0.25, 1)]:
        u = np.log(rng.random(nv * W * H)) * 3.0
        s = rng.integers(0, 256, (nv * W * H + 7) // 8).astype(np.uint8)
        out_s, signs_out = R.log_convolve_signed(W, H, g, u, s, nv)
        save(f"logconv_{W}x{H}_g{g}", W=W, H=H, gamma=g, nv=nv, u=u, out=R.log_convolve(W, H, g, u, nv),
             signs_in=s, out_signed=out_s, signs_out=signs_out)

    # Losses (cpp/loss.h).
    v1 = blob_histograms(1, 10, 9, seed=5)[0]
    v2 = blob_histograms(1, 10, 9, seed=6)[0]
    losses = {}
    for lt in (1, 2, 3, 4):
        f, gr = R.loss(lt, 10, 9, 2.0, v1, v2)
        losses[f"f{lt}"], losses[f"g{lt}"] = f, gr
    save("loss_10x9", W=10, H=9, gamma=2.0, v1=v1, v2=v2, **losses)

    # compute_gradient_both for one histogram, every loss (cpp/inverseWasserstein.h:544-674).
    for (W, H, D, K, L, g, lt) in [(8, 8, 1, 2, 3, 2.0, 2), (16, 12, 1, 3, 10, 2.0, 1),
                                   (16, 12, 1, 3, 10, 2.0, 2), (16, 12, 1, 3, 10, 1.0, 4),
                                   (12, 10, 1, 2, 6, 2.0, 3), (6, 5, 4, 2, 5, 2.0, 2)]:
        N = W * H * D
        obs = blob_histograms(1, W, H, D, seed=11)[0]
        atoms = init_atoms(K, N, seed=12)
        lam = init_weights(1, K, seed=13)[0]
        la, dic, bary = R.gradient_both(W, H, D, g, K, L, lt, atoms, lam, obs)
        save(f"grad_{W}x{H}x{D}_K{K}_L{L}_loss{lt}", W=W, H=H, D=D, K=K, L=L, gamma=g, loss=lt,
             atoms=atoms, lambdas=lam, obs=obs, resultLa=la, resultDic=dic, bary=bary)

    # Log-domain gradient (cpp/inverseWasserstein.h:678-814).
    for (W, H, K, L, g, lt) in [(12, 10, 3, 6, 0.5, 1), (16, 16, 2, 8, 1.0, 4)]:
        N = W * H
        obs = blob_histograms(1, W, H, seed=21, std_frac=(0.01, 0.04))[0]
        atoms = init_atoms(K, N, seed=22)
        lam = init_weights(1, K, seed=23)[0]
        la, dic, bary = R.gradient_both_log(W, H, g, K, L, lt, atoms, lam, obs)
        save(f"gradlog_{W}x{H}_K{K}_L{L}_loss{lt}", W=W, H=H, K=K, L=L, gamma=g, loss=lt,
             atoms=atoms, lambdas=lam, obs=obs, resultLa=la, resultDic=dic, bary=bary)

    # Barycenters (cpp/inverseWasserstein.h:115-201).
    for (W, H, D, K, L, g, log) in [(16, 16, 1, 3, 20, 2.0, False), (12, 12, 1, 3, 15, 0.5, True),
                                    (6, 6, 6, 2, 10, 2.0, False)]:
        N = W * H * D
        atoms = blob_histograms(K, W, H, D, seed=31)
        lam = init_weights(1, K, seed=32)[0]
        bary = R.barycenter(W, H, D, g, K, L, atoms, lam, log_domain=log)
        save(f"bary_{W}x{H}x{D}_K{K}_L{L}_{'log' if log else 'ker'}", W=W, H=H, D=D, K=K, L=L,
             gamma=g, log=log, atoms=atoms, lambdas=lam, bary=bary)

    # evaluate_both over P histograms (cpp/inverseWasserstein.h:986-1145).
    for (P, W, H, D, K, L, g, lt, log) in [(3, 16, 16, 1, 3, 10, 2.0, 2, False),
                                           (4, 16, 12, 1, 3, 12, 1.0, 4, False),
                                           (2, 12, 12, 1, 2, 8, 2.0, 1, False),
                                           (2, 6, 5, 4, 2, 5, 2.0, 2, False),
                                           (2, 12, 12, 1, 3, 8, 0.5, 1, True)]:
        N = W * H * D
        obs = blob_histograms(P, W, H, D, seed=41)
        atoms = init_atoms(K, N, seed=42)
        w = init_weights(P, K, seed=43)
        sd = scale_dictionary(N, P)
        x = to_variables(w, atoms, sd)
        f, gr = R.evaluate_both(W, H, D, g, P, K, L, lt, sd, x, obs, log_domain=log)
        save(f"eval_P{P}_{W}x{H}x{D}_K{K}_L{L}_loss{lt}_{'log' if log else 'ker'}", P=P, W=W, H=H,
             D=D, K=K, L=L, gamma=g, loss=lt, log=log, scale_dic=sd, x=x, obs=obs, f=f, g=gr)

    # Warm restart (cpp/inverseWasserstein.h:1057-1061, :1081-1085).
    P, W, H, K, L, g = 2, 12, 10, 2, 5, 2.0
    N = W * H
    obs = blob_histograms(P, W, H, seed=51)
    atoms = init_atoms(K, N, seed=52)
    w = init_weights(P, K, seed=53)
    sd = scale_dictionary(N, P)
    x = to_variables(w, atoms, sd)
    bs = 1.0 + 0.5 * rng.random(P * K * N)
    f, gr, bl = R.evaluate_both_warm(W, H, g, P, K, L, 2, sd, x, obs, bs)
    save("warm_P2_12x10_K2_L5", P=P, W=W, H=H, K=K, L=L, gamma=g, loss=2, scale_dic=sd, x=x,
         obs=obs, b_storage=bs, f=f, g=gr, b_last=bl)

    # A few L-BFGS iterations of regress_both (cpp/inverseWasserstein.h:362-521).
    P, W, H, K, L, g, iters = 3, 12, 12, 2, 5, 2.0, 4
    N = W * H
    obs = blob_histograms(P, W, H, seed=61)
    atoms = init_atoms(K, N, seed=62)
    w = init_weights(P, K, seed=63)
    sd = scale_dictionary(N, P)
    sol0 = np.concatenate([w.reshape(-1), atoms.reshape(-1)])
    sol = R.regress_both(W, H, g, P, K, L, 2, sd, iters, sol0, obs)
    save("regress_P3_12x12_K2_L5_it4", P=P, W=W, H=H, K=K, L=L, gamma=g, loss=2, scale_dic=sd,
         iters=iters, obs=obs, solution0=sol0, solution=sol)


if __name__ == "__main__":
    main()
