"""Many independent problems per launch (wdl_batch_run) and the uneven
weight-fitting driver built on it.

`batch_run` sends a list of problems (each its own grid side <= 128, K, L, P
and mode) to one persistent launch of the fused tensor-core kernel.

`fit_device` (wdl_fit_weights) fits the barycentric weights of many
histograms against their own fixed dictionaries (the weight half of
regress_both with the atoms held fixed, cpp/inverseWasserstein.h:362-521,
:635-673) with the L-BFGS on the device: every round evaluates all active
histograms of all problems in ONE launch and advances every optimisation in
a second kernel, the round replayed as a CUDA graph.

`fit_weights` is the uneven-workload driver around it: problems of sides up to
128 go to the kernel-domain device fit per gamma; problems above the tile, and
problems whose kernel-domain scalings overflow, go to the log-domain fit
(wdl_fit_weights_log: one persistent launch per gamma, every fit wholly on the
device).  `_fit_host` keeps the host-driven form (host L-BFGS around the
operator path), the reference's control flow, for comparison.
"""
from __future__ import annotations

import ctypes as C
from collections import defaultdict
from concurrent.futures import ThreadPoolExecutor

import numpy as np

from . import lbfgs as lb
from ._lib import (WDL_FIT_OVERFLOW, WDL_MODE_BARYCENTER, WDL_MODE_BOTH, WDL_MODE_WEIGHTS,
                   WdlFitProblem, WdlProblem, check, dptr, f64, lib)
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


def fit_device(kernel, problems, lbfgs_iterations=40, epsilon=1e-50, log_domain=False):
    """wdl_fit_weights: every histogram of every problem fitted by its own
    L-BFGS on the device, all evaluated together each round.  problems: dicts
    with W, H, K, L, atoms [K*N], observed [P*N] (P = len / N), loss_type,
    optional x0 [P*K].  Returns per problem (weights [P,K], loss [P], status
    [P], evaluations [P]).  log_domain: wdl_fit_weights_log on a log-domain
    kernel (one persistent launch, each fit wholly on the device).  epsilon:
    the L-BFGS gradient test; the default 1e-50 is regress_both's setting
    (cpp/inverseWasserstein.h:366), so every fit runs its full iteration
    budget unless its line search stops it."""
    n = len(problems)
    arr = (WdlFitProblem * n)()
    keep, outs = [], []
    for i, pr in enumerate(problems):
        W, H, K, L = (int(pr[k]) for k in ("W", "H", "K", "L"))
        N = W * H
        atoms = f64(pr["atoms"]).reshape(-1)
        obs = f64(pr["observed"]).reshape(-1)
        P = obs.size // N
        x0 = None if pr.get("x0") is None else f64(pr["x0"]).reshape(-1)
        w, f = np.empty(P * K), np.empty(P)
        st, ev = np.empty(P, dtype=np.int32), np.empty(P, dtype=np.int32)
        keep += [atoms, obs, x0]
        outs.append((w, f, st, ev, P, K))
        arr[i] = WdlFitProblem(W, H, K, L, P, int(pr.get("loss_type", 2)), dptr(atoms), dptr(obs),
                               dptr(x0), dptr(w), dptr(f), st.ctypes.data_as(C.POINTER(C.c_int)),
                               ev.ctypes.data_as(C.POINTER(C.c_int)))
    fn = lib().wdl_fit_weights_log if log_domain else lib().wdl_fit_weights
    check(fn(kernel.ctx, C.cast(arr, C.c_void_p), n, int(lbfgs_iterations), float(epsilon)), kernel.ctx)
    return [(w.reshape(P, K), f, st, ev) for (w, f, st, ev, P, K) in outs]


def fit_weights(problems, precision="split_bf16", lbfgs_iterations=40, device=0, max_side=128,
                epsilon=1e-50):
    """problems: dicts with W, H, K, L, gamma, atoms [K*N], observed [N],
    loss_type.  Returns per problem (weights [K], loss, lbfgs status,
    evaluations, domain).

    Problems whose side fits the tensor-core tile are fitted in the kernel
    domain on the device, all problems of a gamma in one wdl_fit_weights call
    (L-BFGS on the device, one fused launch per round).  The kernel domain's
    scalings grow with the iterations when the atoms put their mass in
    different places (they tend to exp(d^2 / gamma) for transport distances
    d, far beyond any float range for a narrow kernel and long runs); a problem
    whose kernel-domain evaluation comes back non-finite is fitted again from
    its start in the log domain (the reference's LogSignArray kernels,
    cpp/kernels.h:1034).  Problems with a side above the tile go to the log
    domain directly.  The log-domain fits of a gamma run as ONE persistent
    launch (wdl_fit_weights_log), every fit wholly on the device."""
    results = [None] * len(problems)
    logq = defaultdict(list)      # gamma -> [(index, evaluations already spent)]
    by_gamma = defaultdict(list)
    for i, pr in enumerate(problems):
        if max(pr["W"], pr["H"]) <= max_side:
            by_gamma[pr["gamma"]].append(i)
        else:
            logq[pr["gamma"]].append((i, 0))
    for g, idx in by_gamma.items():
        kern = CudaGaussian2DKernel(g, max_side, max_side, precision=precision, device=device)
        try:
            outs = fit_device(kern, [problems[i] for i in idx], lbfgs_iterations, epsilon)
        finally:
            kern.close()
        for i, (w, f, st, ev) in zip(idx, outs):
            if int(st[0]) == WDL_FIT_OVERFLOW:
                logq[g].append((i, int(ev[0])))
            else:
                results[i] = (w[0], float(f[0]), int(st[0]), int(ev[0]), "kernel")
    def log_fit(item):
        g, todo = item
        side = max(max(problems[i]["W"], problems[i]["H"]) for i, _ in todo)
        kern = CudaLogSignArrayGaussian2DKernel(g, side, side, precision="fp32", device=device)
        try:
            return fit_device(kern, [problems[i] for i, _ in todo], lbfgs_iterations, epsilon,
                              log_domain=True)
        finally:
            kern.close()

    # one context (and stream) per gamma; the library calls release the
    # interpreter lock, so the gammas' launches run concurrently on the GPU
    items = list(logq.items())
    with ThreadPoolExecutor(max_workers=max(1, len(items))) as ex:
        outs_all = list(ex.map(log_fit, items))
    for (g, todo), outs in zip(items, outs_all):
        for (i, spent), (w, f, st, ev) in zip(todo, outs):
            results[i] = (w[0], float(f[0]), int(st[0]), int(ev[0]) + spent, "log")
    return results


def _fit_host(problems, todo, lbfgs_iterations, device, epsilon):
    """Host L-BFGS per problem (resumable generator), every round's
    evaluations issued problem by problem on the operator path of each
    problem's grid: FP32 kernel domain, or the log domain."""
    param = lb.LbfgsParam(max_iterations=lbfgs_iterations, epsilon=epsilon)
    states = []
    for i, dom, _ in todo:
        gen = lb.lbfgs_steps(np.zeros(int(problems[i]["K"])), param)
        states.append({"i": i, "gen": gen, "x": next(gen), "done": False, "evals": 0, "seen": {},
                       "domain": dom})
    ctxs = {}

    def ctx_for(key):
        if key not in ctxs:
            kind, W, H, g = key
            if kind == "kernel":
                ctxs[key] = CudaGaussian2DKernel(g, W, H, precision="fp32", device=device)
            else:
                ctxs[key] = CudaLogSignArrayGaussian2DKernel(g, W, H, precision="fp32", device=device)
        return ctxs[key]

    results = [None] * len(states)
    try:
        while True:
            active = [j for j, s in enumerate(states) if not s["done"]]
            if not active:
                break
            for j in active:
                s = states[j]
                pr = problems[s["i"]]
                kern = ctx_for((s["domain"], pr["W"], pr["H"], pr["gamma"]))
                x = s["x"]
                w = np.exp(x - x.max())
                w /= w.sum()
                K, N = int(pr["K"]), pr["W"] * pr["H"]
                la, dic, loss = np.empty(K), np.empty(K * N), np.empty(1)
                check(lib().wdl_gradient_both(kern.ctx, 1, K, int(pr["L"]), int(pr.get("loss_type", 2)),
                                              dptr(f64(pr["atoms"])), dptr(w), dptr(f64(pr["observed"])),
                                              None, dptr(la), dptr(dic), None, dptr(loss), None),
                      kern.ctx)
                f = float(loss[0])
                finite = np.isfinite(f) and np.all(np.isfinite(la))
                if not finite and s["domain"] == "kernel":
                    s["domain"] = "log"  # re-evaluate the same point next round
                    continue
                s["evals"] += 1
                g = (la - np.dot(w, la)) * w
                if not finite:
                    f, g = float("inf"), np.zeros_like(g)
                s["seen"][x.tobytes()] = f
                try:
                    s["x"] = s["gen"].send((f, g))
                except StopIteration as e:
                    # a failed line search returns the last accepted point with
                    # the last TRIAL value (as liblbfgs does): report the loss
                    # evaluated at the point returned
                    status, xr, fx = e.value
                    wr = np.exp(xr - xr.max())
                    results[j] = (wr / wr.sum(), s["seen"].get(xr.tobytes(), fx), status, s["evals"],
                                  s["domain"])
                    s["done"] = True
    finally:
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
