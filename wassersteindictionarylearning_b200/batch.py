"""Many independent problems per launch (wdl_batch_run) and the uneven
weight-fitting driver built on it.

`batch_run` sends a list of problems (each its own grid side <= 128, K, L, P
and mode) to one persistent launch of the fused tensor-core kernel.

`fit_weights` fits the barycentric weights of many single histograms against
their own fixed dictionaries (the weight half of regress_both with the atoms
held fixed, cpp/inverseWasserstein.h:362-521, :635-673): every problem runs its
own resumable L-BFGS (lbfgs.lbfgs_steps, liblbfgs' parameters); each round,
all active problems of a gamma are evaluated in ONE batched launch on that
gamma's context.  Problems with a side above 128 are evaluated on the FP32
operator path of their own grid, and problems whose kernel-domain scalings
overflow move to the log-domain operator.
"""
from __future__ import annotations

import ctypes as C
from collections import defaultdict

import numpy as np

from . import lbfgs as lb
from ._lib import (WDL_MODE_BARYCENTER, WDL_MODE_BOTH, WDL_MODE_WEIGHTS, WdlProblem, check, dptr,
                   f64, lib)
from .kernels import CudaGaussian2DKernel, CudaLogSignArrayGaussian2DKernel

MODES = {"weights": WDL_MODE_WEIGHTS, "both": WDL_MODE_BOTH, "barycenter": WDL_MODE_BARYCENTER}


def batch_run(kernel, problems):
    """problems: dicts with W, H, K, L, P, atoms [K*N], weights [P*K], and for
    gradient modes observed [P*N] and loss_type; mode in MODES.  Returns per
    problem a dict with la, dic, bary, loss (as the mode provides)."""
    n = len(problems)
    arr = (WdlProblem * n)()
    keep, outs = [], []
    for i, pr in enumerate(problems):
        W, H, K, L, P = (int(pr[k]) for k in ("W", "H", "K", "L", "P"))
        N = W * H
        mode = MODES[pr.get("mode", "weights")]
        atoms = f64(pr["atoms"]).reshape(-1)
        weights = f64(pr["weights"]).reshape(-1)
        obs = None if mode == WDL_MODE_BARYCENTER else f64(pr["observed"]).reshape(-1)
        o = {}
        if mode != WDL_MODE_BARYCENTER:
            o["la"] = np.empty(P * K)
            o["loss"] = np.empty(P)
        if mode == WDL_MODE_BOTH:
            o["dic"] = np.empty(K * N)
        if mode == WDL_MODE_BARYCENTER or pr.get("want_bary"):
            o["bary"] = np.empty(P * N)
        keep += [atoms, weights, obs]
        outs.append(o)
        arr[i] = WdlProblem(W, H, K, L, P, int(pr.get("loss_type", 2)), mode, dptr(atoms),
                            dptr(weights), dptr(obs), dptr(o.get("la")), dptr(o.get("dic")),
                            dptr(o.get("bary")), dptr(o.get("loss")))
    check(lib().wdl_batch_run(kernel.ctx, C.cast(arr, C.c_void_p), n), kernel.ctx)
    return outs


def fit_weights(problems, precision="split_bf16", lbfgs_iterations=40, device=0, max_side=128):
    """problems: dicts with W, H, K, L, gamma, atoms [K*N], observed [N],
    loss_type.  Returns per problem (weights [K], loss, lbfgs status,
    evaluations, domain).

    Every problem starts in the kernel domain, batched per gamma.  The kernel
    domain's scalings grow with the iterations wherever the atoms are nearly
    empty (the dual potentials reach |d|^2 / gamma, far beyond any float range
    for peaked atoms, a narrow kernel and long runs); a problem whose
    evaluation comes back non-finite is moved, at the same point, to the
    log-domain operator (the reference's LogSignArray kernels,
    cpp/kernels.h:1034) and stays there."""
    param = lb.LbfgsParam(max_iterations=lbfgs_iterations, epsilon=1e-6)
    states = []
    for pr in problems:
        gen = lb.lbfgs_steps(np.zeros(int(pr["K"])), param)
        states.append({"gen": gen, "x": next(gen), "done": False, "evals": 0, "seen": {},
                       "domain": "kernel"})
    ctxs = {}

    def ctx_for(key):
        if key not in ctxs:
            kind, W, H, g = key
            if kind == "tc":
                ctxs[key] = CudaGaussian2DKernel(g, W, H, precision=precision, device=device)
            elif kind == "kernel":
                ctxs[key] = CudaGaussian2DKernel(g, W, H, precision="fp32", device=device)
            else:
                ctxs[key] = CudaLogSignArrayGaussian2DKernel(g, W, H, precision="fp32", device=device)
        return ctxs[key]

    results = [None] * len(problems)
    while True:
        active = [i for i, s in enumerate(states) if not s["done"]]
        if not active:
            break
        groups = defaultdict(list)
        for i in active:
            pr = problems[i]
            if states[i]["domain"] == "log":
                key = ("log", pr["W"], pr["H"], pr["gamma"])
            elif max(pr["W"], pr["H"]) > max_side:
                key = ("kernel", pr["W"], pr["H"], pr["gamma"])
            else:
                key = ("tc", max_side, max_side, pr["gamma"])
            groups[key].append(i)
        evals = {}
        for key, idx in groups.items():
            lam = {}
            batch = []
            for i in idx:
                x = states[i]["x"]
                w = np.exp(x - x.max())
                lam[i] = w / w.sum()
                pr = problems[i]
                batch.append(dict(W=pr["W"], H=pr["H"], K=pr["K"], L=pr["L"], P=1, atoms=pr["atoms"],
                                  weights=lam[i], observed=pr["observed"],
                                  loss_type=pr.get("loss_type", 2), mode="weights"))
            kern = ctx_for(key)
            if key[0] == "tc":
                outs = batch_run(kern, batch)
            else:  # one problem per call on the operator path of its own grid
                outs = []
                for b in batch:
                    K, N = b["K"], b["W"] * b["H"]
                    la, dic, loss = np.empty(K), np.empty(K * N), np.empty(1)
                    check(lib().wdl_gradient_both(kern.ctx, 1, K, b["L"], b["loss_type"],
                                                  dptr(f64(b["atoms"])), dptr(f64(b["weights"])),
                                                  dptr(f64(b["observed"])), None, dptr(la),
                                                  dptr(dic), None, dptr(loss), None), kern.ctx)
                    outs.append({"la": la, "loss": loss})
            for i, o in zip(idx, outs):
                evals[i] = (o, lam[i])
        for i, (o, w) in evals.items():
            s = states[i]
            la = o["la"]
            f = float(o["loss"][0])
            finite = np.isfinite(f) and np.all(np.isfinite(la))
            if not finite and s["domain"] == "kernel":
                s["domain"] = "log"  # re-evaluate the same point next round
                continue
            s["evals"] += 1
            g = (la - np.dot(w, la)) * w
            if not finite:
                f, g = float("inf"), np.zeros_like(g)
            s["seen"][s["x"].tobytes()] = f
            try:
                s["x"] = s["gen"].send((f, g))
            except StopIteration as e:
                # a failed line search returns the last accepted point with
                # the last TRIAL value (as liblbfgs does): report the loss
                # evaluated at the point returned
                status, x, fx = e.value
                w = np.exp(x - x.max())
                results[i] = (w / w.sum(), s["seen"].get(x.tobytes(), fx), status, s["evals"],
                              s["domain"])
                s["done"] = True
    for k in ctxs.values():
        k.close()
    return results


def uneven_problems(n=512, seed=0, sides=(32, 48, 64, 96, 128, 192), K_range=(3, 8),
                    L_range=(25, 100), gammas=(1.0, 2.0, 4.0)):
    """The uneven weight-fitting workload: per problem a side from `sides`, K
    uniform in K_range, L uniform in L_range, gamma from `gammas`, a fixed
    random-blob dictionary, and an observation that is a blob histogram."""
    from .synthetic import blob_histograms
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for i in range(n):
        side = int(rng.choice(sides))
        K = int(rng.integers(K_range[0], K_range[1] + 1))
        L = int(rng.integers(L_range[0], L_range[1] + 1))
        g = float(rng.choice(gammas))
        atoms = blob_histograms(K, side, side, seed=seed * 7919 + 2 * i)
        obs = blob_histograms(1, side, side, seed=seed * 7919 + 2 * i + 1)[0]
        out.append(dict(W=side, H=side, K=K, L=L, gamma=g, atoms=atoms.reshape(-1), observed=obs,
                        loss_type=2))
    return out
