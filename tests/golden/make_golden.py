"""Generate the golden fixtures in this folder from the reference's own code.

Runs the UNMODIFIED reference (compiled by oracle/Makefile into oracle/_ref from
the reference sources) on small seeded inputs and stores inputs and outputs as
compressed .npz files.  The reference ships no tests or fixtures of its own, so
these runs are what pins the oracle and the CUDA path.

    python tests/golden/make_golden.py           # needs oracle/_ref (reference sources present)
    python tests/golden/make_golden.py --large   # only the full-grid fixtures (minutes of CPU)

The full-grid fixtures (256x256 log domain, 48^3 kernel domain) do not store
their inputs: the tests regenerate them from the recorded seeds with
wassersteindictionarylearning_b200.synthetic and check a few input statistics
(``in_stats``) first.  Their large outputs are stored as every STRIDE-th entry
plus the entry count, maximum magnitude, sum and sum of magnitudes of the whole
array (``sample_stats``), which keeps each fixture well under a megabyte.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.oracle import OracleLib, RefLib  # noqa: E402
from wassersteindictionarylearning_b200.synthetic import (blob_histograms, init_atoms,  # noqa: E402
                                                          init_weights, scale_dictionary,
                                                          to_variables)


def save(name, **arrays):
    path = os.path.join(HERE, name + ".npz")
    np.savez_compressed(path, **{k: np.asarray(v) for k, v in arrays.items()})
    print("wrote", path, os.path.getsize(path), "bytes")


STRIDE = 16


def sample_stats(a, stride=STRIDE):
    a = np.asarray(a, dtype=np.float64).reshape(-1)
    return dict(sample=a[::stride].copy(), n=a.size, absmax=float(np.max(np.abs(a))),
                total=float(np.sum(a)), abssum=float(np.sum(np.abs(a))), stride=stride)


def in_stats(*arrays):
    return np.array([v for a in arrays for v in (float(np.sum(a)), float(np.sum(np.asarray(a) ** 2)),
                                                  float(np.max(a)), float(np.min(a)))])


def save_stats(name, prefix, a, out):
    for k, v in sample_stats(a).items():
        out[f"{prefix}_{k}"] = v


def large():
    """Full-grid fixtures: the log-domain configuration's grid (256x256, K=8,
    gamma 0.5, TV loss, 1-3 sharp blobs of std 0.01-0.04 of the side) at the
    reduced P and L of a CPU run, its signed operator alone, and the serving
    volume (48^3, K=5, L=50, gamma 2) in the kernel domain."""
    R = RefLib()
    O = OracleLib()  # condition scales of the weight gradients (the reference has no such output)
    # compute_gradient_both_log_signArray (cpp/inverseWasserstein.h:678-814), one histogram
    W = H = 256
    N = W * H
    K, L, g, lt = 8, 10, 0.5, 1
    obs = blob_histograms(1, W, H, n_blobs=(1, 3), std_frac=(0.01, 0.04), seed=71)[0]
    atoms = init_atoms(K, N, seed=72)
    lam = init_weights(1, K, seed=73)[0]
    la, dic, bary = R.gradient_both_log(W, H, g, K, L, lt, atoms, lam, obs)
    out = dict(W=W, H=H, K=K, L=L, gamma=g, loss=lt, seeds=np.array([71, 72, 73]),
               in_stats=in_stats(obs, atoms, lam), lambdas=lam, resultLa=la, bary=bary,
               resultLa_scale=O.gradient_both_scale(W, H, 1, g, K, L, lt, atoms, lam, obs, log_domain=True))
    save_stats("gradlog_256x256_K8_L10_loss1", "resultDic", dic, out)
    save("full_gradlog_256x256_K8_L10_loss1", **out)

    # evaluate_both in the log domain over P = 2 histograms (:986-1145)
    P = 2
    obs = blob_histograms(P, W, H, n_blobs=(1, 3), std_frac=(0.01, 0.04), seed=81)
    atoms = init_atoms(K, N, seed=82)
    w = init_weights(P, K, seed=83)
    sd = scale_dictionary(N, P)
    x = to_variables(w, atoms, sd)
    f, gr = R.evaluate_both(W, H, 1, g, P, K, L, lt, sd, x, obs, log_domain=True)
    out = dict(P=P, W=W, H=H, K=K, L=L, gamma=g, loss=lt, scale_dic=sd, seeds=np.array([81, 82, 83]),
               in_stats=in_stats(obs, atoms, w), f=f, g_weights=gr[:P * K],
               g_weights_scale=O.weight_gradient_scale(W, H, 1, g, P, K, L, lt, sd, x, obs, log_domain=True))
    save_stats("eval_P2_256x256_K8_L10_loss1_log", "g_atoms", gr[P * K:], out)
    save("full_eval_P2_256x256_K8_L10_loss1_log", **out)

    # log_convolve and log_convolve_signArray alone (cpp/kernels.h:1073-1163)
    rng = np.random.Generator(np.random.PCG64(91))
    u = np.log(rng.random(N)) * 3.0
    sg = rng.integers(0, 256, (N + 7) // 8).astype(np.uint8)
    out_s, signs_out = R.log_convolve_signed(W, H, g, u, sg, 1)
    out = dict(W=W, H=H, gamma=g, nv=1, seed=91, in_stats=in_stats(u), signs_in=sg, signs_out=signs_out)
    save_stats("logconv_256x256_g0.5", "out", R.log_convolve(W, H, g, u, 1), out)
    save_stats("logconv_256x256_g0.5", "out_signed", out_s, out)
    save("full_logconv_256x256_g0.5", **out)

    # the serving volume in the kernel domain: compute_gradient_both on 48^3 (Gaussian3DKernel)
    W = H = D = 48
    N = W * H * D
    K, L, g, lt = 5, 50, 2.0, 2
    obs = blob_histograms(1, W, H, D, n_blobs=(1, 3), std_frac=(0.05, 0.12), seed=101)[0]
    atoms = init_atoms(K, N, seed=102)
    lam = init_weights(1, K, seed=103)[0]
    la, dic, bary = R.gradient_both(W, H, D, g, K, L, lt, atoms, lam, obs)
    out = dict(W=W, H=H, D=D, K=K, L=L, gamma=g, loss=lt, seeds=np.array([101, 102, 103]),
               in_stats=in_stats(obs, atoms, lam), lambdas=lam, resultLa=la,
               resultLa_scale=O.gradient_both_scale(W, H, D, g, K, L, lt, atoms, lam, obs))
    save_stats("grad_48x48x48_K5_L50_loss2", "bary", bary, out)
    save_stats("grad_48x48x48_K5_L50_loss2", "resultDic", dic, out)
    save("full_grad_48x48x48_K5_L50_loss2", **out)


def main():
    if "--large" in sys.argv:
        large()
        return
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
