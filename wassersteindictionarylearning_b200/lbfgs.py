"""Host L-BFGS with the semantics the reference's driver relies on.

Restates the limited-memory BFGS of liblbfgs 1.10 (the library vendored at
cpp/lbfgs/lbfgs.c) for the configuration WassersteinRegression::regress_both
uses (cpp/inverseWasserstein.h:365-372): m = 6 correction pairs, the two-loop
recursion for the direction (Nocedal 1980; lbfgs.c:570-612), and the
backtracking line search with the strong Wolfe test (lbfgs.c:772-867:
step x0.5 on failure of sufficient decrease or of the curvature bound, x2.1 when
the directional derivative is still too negative, ftol 1e-4, wolfe 0.9, at most
20 trials, step bounds 1e-20..1e20), and the stopping rules of lbfgs.c:256-654
(gradient test |g|/max(1,|x|) <= epsilon, max_iterations accepted steps).
Return codes use liblbfgs' values (cpp/lbfgs/lbfgs.h:74-147).
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Callable, Optional

import numpy as np

LBFGS_SUCCESS = 0
LBFGS_STOP = 1
LBFGS_ALREADY_MINIMIZED = 2
LBFGSERR_UNKNOWNERROR = -1024
LBFGSERR_CANCELED = -1021
LBFGSERR_MINIMUMSTEP = -1000
LBFGSERR_MAXIMUMSTEP = -999
LBFGSERR_MAXIMUMLINESEARCH = -998
LBFGSERR_MAXIMUMITERATION = -997
LBFGSERR_INVALIDPARAMETERS = -995
LBFGSERR_INCREASEGRADIENT = -994


@dataclass
class LbfgsParam:
    m: int = 6
    epsilon: float = 1e-50
    past: int = 0
    delta: float = 1e-50
    max_iterations: int = 0
    max_linesearch: int = 20
    min_step: float = 1e-20
    max_step: float = 1e20
    ftol: float = 1e-4
    wolfe: float = 0.9


Evaluate = Callable[[np.ndarray, float], tuple]        # (x, step) -> (f, g)
Progress = Callable[[np.ndarray, np.ndarray, float, float, float, float, int, int], int]


def _minimize(x0: np.ndarray, p: LbfgsParam, progress: Optional[Progress], nan_cancel: bool,
              state: dict):
    """The algorithm, once: a generator that yields each point to evaluate and
    receives (f, g) through send(); it returns (status, x, f) via StopIteration.
    state["step"] holds the line-search step of the point being evaluated (0
    for the first evaluation).  progress, when given, is called after every
    accepted step (lbfgs.c:522-529) and a non-zero return stops the run; with
    nan_cancel a NaN objective stops it instead (LBFGSERR_CANCELED, the
    reference's progress_both, cpp/inverseWasserstein.h:1180-1184)."""
    x = np.array(x0, dtype=np.float64, copy=True)
    n = x.size
    state["step"] = 0.0
    f, g = yield x
    g = np.asarray(g, dtype=np.float64)
    d = -g
    xnorm = max(float(np.linalg.norm(x)), 1.0)
    gnorm = float(np.linalg.norm(g))
    if gnorm / xnorm <= p.epsilon:
        return LBFGS_ALREADY_MINIMIZED, x, f
    step = 1.0 / float(np.sqrt(np.dot(d, d)))
    s_hist = np.zeros((p.m, n))
    y_hist = np.zeros((p.m, n))
    ys_hist = np.zeros(p.m)
    alpha = np.zeros(p.m)
    pf = np.zeros(max(p.past, 1))
    if p.past > 0:
        pf[0] = f
    k, end = 1, 0
    while True:
        xp, gp = x.copy(), g.copy()
        # backtracking line search with the strong Wolfe test (lbfgs.c:772-867);
        # on failure the run stops at the previous point (lbfgs.c:487-492)
        if step <= 0:
            return LBFGSERR_INVALIDPARAMETERS, xp, f
        dginit = float(np.dot(g, d))
        if dginit > 0:
            return LBFGSERR_INCREASEGRADIENT, xp, f
        finit, dgtest, count = f, p.ftol * dginit, 0
        while True:
            x = xp + step * d
            state["step"] = step
            f, g = yield x
            g = np.asarray(g, dtype=np.float64)
            count += 1
            if f > finit + step * dgtest:
                width = 0.5
            else:
                dg = float(np.dot(g, d))
                if dg < p.wolfe * dginit:
                    width = 2.1
                elif dg > -p.wolfe * dginit:
                    width = 0.5
                else:
                    break
            if step < p.min_step:
                return LBFGSERR_MINIMUMSTEP, xp, f
            if step > p.max_step:
                return LBFGSERR_MAXIMUMSTEP, xp, f
            if p.max_linesearch <= count:
                return LBFGSERR_MAXIMUMLINESEARCH, xp, f
            step *= width
        xnorm = float(np.linalg.norm(x))
        gnorm = float(np.linalg.norm(g))
        if progress is not None:
            ret = progress(x, g, f, xnorm, gnorm, step, k, count)
            if ret:
                return ret, x, f
        if nan_cancel and np.isnan(f):
            return LBFGSERR_CANCELED, x, f
        if gnorm / max(xnorm, 1.0) <= p.epsilon:
            return LBFGS_SUCCESS, x, f
        if p.past > 0:
            if p.past <= k:
                rate = (pf[k % p.past] - f) / f
                if rate < p.delta:
                    return LBFGS_STOP, x, f
            pf[k % p.past] = f
        if p.max_iterations != 0 and p.max_iterations < k + 1:
            return LBFGSERR_MAXIMUMITERATION, x, f
        # two-loop recursion over the m most recent pairs (lbfgs.c:570-612)
        s_hist[end] = x - xp
        y_hist[end] = g - gp
        ys = float(np.dot(y_hist[end], s_hist[end]))
        yy = float(np.dot(y_hist[end], y_hist[end]))
        ys_hist[end] = ys
        bound = min(p.m, k)
        k += 1
        end = (end + 1) % p.m
        d = -g
        j = end
        for _ in range(bound):
            j = (j + p.m - 1) % p.m
            alpha[j] = float(np.dot(s_hist[j], d)) / ys_hist[j]
            d = d - alpha[j] * y_hist[j]
        d = d * (ys / yy)
        for _ in range(bound):
            beta = float(np.dot(y_hist[j], d)) / ys_hist[j]
            d = d + (alpha[j] - beta) * s_hist[j]
            j = (j + 1) % p.m
        step = 1.0


def lbfgs_steps(x0: np.ndarray, param: Optional[LbfgsParam] = None):
    """Resumable form: a generator that yields each point to evaluate and
    receives (f, g) through send(); it returns (status, x, f) via StopIteration.
    A NaN objective cancels the run as the reference's progress_both does."""
    return _minimize(x0, param or LbfgsParam(), None, True, {})


def lbfgs(x0: np.ndarray, evaluate: Evaluate, progress: Optional[Progress] = None,
          param: Optional[LbfgsParam] = None):
    """Minimise f from x0 with evaluate(x, step) -> (f, g) and the optional
    progress callback (liblbfgs' lbfgs(), lbfgs.c:256-654).  Returns (status, x, f)."""
    state = {}
    gen = _minimize(x0, param or LbfgsParam(), progress, False, state)
    try:
        x = next(gen)
        while True:
            x = gen.send(evaluate(x, state["step"]))
    except StopIteration as stop:
        return stop.value
