"""Continuous-batching request loop for barycenter and projection requests.

Two request kinds, both against a resident dictionary of K atoms per grid shape:

* barycenter: given weights, the forward Bregman projections
  (WassersteinBarycenter::compute_barycenter, cpp/inverseWasserstein.h:115-153);
* projection: fit the K barycentric weights of one new histogram, i.e. minimise
  loss(bary(w), obs) over w on the simplex with L-BFGS — the weight half of
  compute_gradient_both (:635-673) with the atoms held fixed.

The engine keeps a device context per grid shape (LRU-bounded), admits pending
requests while the HBM bytes of the admitted requests' iterate stores fit the
budget, and runs in ticks: every tick, each shape's active requests go to the
device as ONE batched call (all barycenter requests of the shape in one
wdl_barycenter call, one objective evaluation for every active projection in one
wdl_gradient_both call).  Shapes run concurrently on their own contexts' streams
from a thread pool.  A projection request carries a resumable L-BFGS
(lbfgs.lbfgs_steps), so requests that arrive while others are on the device join
at the next tick and leave as soon as their optimisation ends.
"""
from __future__ import annotations

import concurrent.futures as cf
import itertools
import threading
import time
from collections import OrderedDict, deque
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import lbfgs as lb
from ._lib import WdlError, check, dptr, f64, lib
from .kernels import CudaGaussian2DKernel, CudaGaussian3DKernel
from .synthetic import blob_histograms

BARYCENTER, PROJECTION = "barycenter", "projection"


@dataclass(eq=False)
class Request:
    kind: str
    shape: tuple                      # (W, H, D)
    weights: Optional[np.ndarray] = None   # barycenter: K weights
    observed: Optional[np.ndarray] = None  # projection: N-pixel histogram
    rid: int = 0
    t_arrival: float = 0.0
    t_admit: float = 0.0
    t_done: float = 0.0
    result: Optional[np.ndarray] = None    # barycenter [N] or fitted weights [K]
    loss: float = float("nan")
    status: int = 0
    lbfgs_status: int = 0   # liblbfgs-style code the projection's optimisation ended with
    bytes: int = 0
    _steps: object = None
    _x: Optional[np.ndarray] = None

    @property
    def latency(self) -> float:
        return self.t_done - self.t_arrival


@dataclass(eq=False)
class _Shape:
    key: tuple
    kernel: object
    atoms: np.ndarray
    active: list = field(default_factory=list)


class ServingEngine:
    """Request loop.  precision: tensor-core form for 2-D shapes up to 512 per
    side (split_bf16 / tf32), FP32 operator path for 3-D shapes."""

    def __init__(self, K: int = 5, L: int = 50, gamma: float = 2.0, loss_type: int = 2,
                 precision: str = "split_bf16", hbm_budget: float = 8e9, max_batch: int = 64,
                 lbfgs_iterations: int = 20, max_shapes: int = 48, workers: int = 8,
                 dictionary_seed: int = 100, device: int = 0):
        self.K, self.L, self.gamma, self.loss_type = K, L, gamma, loss_type
        self.precision = precision
        self.hbm_budget = hbm_budget
        self.max_batch = max_batch
        self.lbfgs_param = lb.LbfgsParam(max_iterations=lbfgs_iterations, epsilon=1e-6)
        self.max_shapes = max_shapes
        self.device = device
        self.dictionary_seed = dictionary_seed
        self._shapes: "OrderedDict[tuple, _Shape]" = OrderedDict()
        self._pending: deque = deque()
        self._lock = threading.Lock()
        self._ids = itertools.count()
        self._pool = cf.ThreadPoolExecutor(max_workers=workers)
        self.admitted_bytes = 0
        self.completed: list = []

    # ---- dictionary / contexts --------------------------------------------------------
    def _precision_for(self, shape):
        # 2-D grids up to 512 take the tensor-core form (fused kernel up to
        # 128, axis-pass GEMMs above); the 48^3 volumes stay FP32 on the CUDA
        # cores, which is faster there (6.7 vs 7.2 ms per evaluation for K=5,
        # L=50: a 48-long axis fills little of a 128 x 64 tensor-core tile)
        W, H, D = shape
        if D == 1 and W <= 512 and H <= 512 and self.precision in ("split_bf16", "tf32"):
            return self.precision
        return "fp32" if self.precision != "fp64" else "fp64"

    def dictionary(self, shape) -> np.ndarray:
        """The resident dictionary of a shape: K seeded blob atoms (fixed per shape)."""
        return self._shape(shape).atoms

    def _shape(self, shape) -> _Shape:
        key = tuple(int(v) for v in shape)
        s = self._shapes.get(key)
        if s is not None:
            self._shapes.move_to_end(key)
            return s
        if len(self._shapes) >= self.max_shapes:  # evict an idle shape (LRU)
            for k2, s2 in list(self._shapes.items()):
                if not s2.active:
                    s2.kernel.close()
                    del self._shapes[k2]
                    break
        W, H, D = key
        prec = self._precision_for(key)
        if D > 1:
            kern = CudaGaussian3DKernel(self.gamma, W, H, D, precision=prec, device=self.device)
        else:
            kern = CudaGaussian2DKernel(self.gamma, W, H, precision=prec, device=self.device)
        seed = self.dictionary_seed + W * 7919 + H * 131 + D
        atoms = blob_histograms(self.K, W, H, D, n_blobs=(1, 3), seed=seed)
        s = _Shape(key, kern, atoms)
        self._shapes[key] = s
        return s

    def request_bytes(self, req: Request) -> int:
        W, H, D = req.shape
        s = self._shape(req.shape)
        L = self.L
        if req.kind == BARYCENTER:
            return int(lib().wdl_eval_bytes(s.kernel.ctx, 1, self.K, 2))
        return int(lib().wdl_eval_bytes(s.kernel.ctx, 1, self.K, L))

    # ---- API -------------------------------------------------------------------------
    def submit(self, req: Request) -> Request:
        req.rid = next(self._ids)
        if not req.t_arrival:
            req.t_arrival = time.perf_counter()
        with self._lock:
            self._pending.append(req)
        return req

    def idle(self) -> bool:
        with self._lock:
            return not self._pending and not any(s.active for s in self._shapes.values())

    def _admit(self):
        with self._lock:
            while self._pending:
                req = self._pending[0]
                if not req.bytes:
                    req.bytes = self.request_bytes(req)
                if req.bytes > self.hbm_budget:
                    self._pending.popleft()
                    req.status = -7  # WDL_ERR_ADMISSION: can never fit
                    req.t_done = time.perf_counter()
                    self.completed.append(req)
                    continue
                if self.admitted_bytes + req.bytes > self.hbm_budget:
                    break
                s = self._shape(req.shape)
                if len(s.active) >= self.max_batch:
                    break
                self._pending.popleft()
                self.admitted_bytes += req.bytes
                req.t_admit = time.perf_counter()
                if req.kind == PROJECTION:
                    x0 = np.zeros(self.K)  # uniform weights
                    req._steps = lb.lbfgs_steps(x0, self.lbfgs_param)
                    req._x = next(req._steps)
                s.active.append(req)

    def _finish(self, s: _Shape, req: Request):
        req.t_done = time.perf_counter()
        s.active.remove(req)
        with self._lock:
            self.admitted_bytes -= req.bytes
            self.completed.append(req)

    # ---- one batched device call per shape ------------------------------------------------
    def _run_shape(self, s: _Shape):
        K, L = self.K, self.L
        ctx = s.kernel.ctx
        N = s.kernel.N
        bary_reqs = [r for r in s.active if r.kind == BARYCENTER]
        proj_reqs = [r for r in s.active if r.kind == PROJECTION]
        if bary_reqs:
            P = len(bary_reqs)
            w = f64(np.stack([r.weights for r in bary_reqs]))
            out = np.empty(P * N)
            rc = lib().wdl_barycenter(ctx, P, K, L, dptr(f64(s.atoms)), dptr(w), dptr(out))
            for i, r in enumerate(bary_reqs):
                r.status = rc
                r.result = out[i * N:(i + 1) * N].copy() if rc == 0 else None
                self._finish(s, r)
        if proj_reqs:
            P = len(proj_reqs)
            # x = log-weights; lambda = normalise(exp(x)) (evaluate_both's transform, :997-1020)
            lam = np.stack([np.exp(r._x - r._x.max()) for r in proj_reqs])
            lam /= lam.sum(axis=1, keepdims=True)
            obs = f64(np.stack([r.observed for r in proj_reqs]))
            la = np.empty(P * K)
            dic = np.empty(K * N)
            loss = np.empty(P)
            rc = lib().wdl_gradient_both(ctx, P, K, L, self.loss_type, dptr(f64(s.atoms)),
                                         dptr(f64(lam)), dptr(obs), None, dptr(la), dptr(dic),
                                         None, dptr(loss), None)
            for i, r in enumerate(proj_reqs):
                if rc != 0:
                    r.status = rc
                    self._finish(s, r)
                    continue
                la_i = la[i * K:(i + 1) * K]
                w_i = lam[i]
                # simplex projection and chain rule of the exp transform (:1093-1098, :1125-1128)
                g = (la_i - np.dot(w_i, la_i)) * w_i
                f_i = float(loss[i])
                if not (np.isfinite(f_i) and np.all(np.isfinite(g))):
                    # A trial point outside the operator's FP32 range: report it as
                    # +inf so the line search halves the step instead of stopping.
                    f_i, g = float("inf"), np.zeros_like(g)
                try:
                    r._x = r._steps.send((f_i, g))
                except StopIteration as e:
                    status, x, f = e.value
                    wts = np.exp(x - x.max())
                    r.result = wts / wts.sum()
                    r.loss = f
                    r.lbfgs_status = status
                    # Like regress_both (cpp/inverseWasserstein.h:413-417), a line-search
                    # or iteration-limit code still returns the last accepted point;
                    # only a cancellation (NaN objective) fails the request.
                    r.status = lb.LBFGSERR_CANCELED if status == lb.LBFGSERR_CANCELED else 0
                    self._finish(s, r)

    def tick(self) -> int:
        """Admit what fits, then one batched call per shape with active requests."""
        self._admit()
        work = [s for s in list(self._shapes.values()) if s.active]
        if not work:
            return 0
        futs = [self._pool.submit(self._run_shape, s) for s in work]
        for f in futs:
            f.result()
        return len(work)

    def run(self, arrivals=None, timeout: float = 600.0):
        """Serve a stream: arrivals is an iterable of (t_offset_s, Request) sorted
        by time; requests are submitted when their time comes, ticks run
        continuously until everything has completed."""
        t0 = time.perf_counter()
        queue = deque(arrivals or [])
        while True:
            now = time.perf_counter() - t0
            while queue and queue[0][0] <= now:
                t_off, req = queue.popleft()
                req.t_arrival = t0 + t_off
                self.submit(req)
            ran = self.tick()
            if not queue and self.idle():
                break
            if not ran and queue:
                time.sleep(min(0.001, max(0.0, queue[0][0] - (time.perf_counter() - t0))))
            if time.perf_counter() - t0 > timeout:
                raise WdlError(-6, "serving run exceeded its timeout")
        return self.completed

    def close(self):
        self._pool.shutdown(wait=True)
        for s in self._shapes.values():
            s.kernel.close()
        self._shapes.clear()


def poisson_requests(rate: float, n: int, seed: int = 0, K: int = 5, frac_3d: float = 0.2,
                     side_range=(64, 256), cube: int = 48, frac_projection: float = 0.5,
                     sides=None):
    """(arrival_offset, Request) pairs: Poisson arrivals at `rate` per second,
    2-D sides uniform in side_range (or drawn from `sides`), a fraction of 3-D
    cube^3 volumes, half projection requests (observed: seeded blob histograms)
    and half barycenter requests (weights: uniform on the simplex)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    t = 0.0
    out = []
    for i in range(n):
        t += rng.exponential(1.0 / rate)
        if rng.random() < frac_3d:
            shape = (cube, cube, cube)
        elif sides is not None:
            s = int(rng.choice(sides))
            shape = (s, s, 1)
        else:
            shape = (int(rng.integers(side_range[0], side_range[1] + 1)),
                     int(rng.integers(side_range[0], side_range[1] + 1)), 1)
        if rng.random() < frac_projection:
            obs = blob_histograms(1, shape[0], shape[1], shape[2], n_blobs=(1, 3),
                                  seed=seed * 100003 + i)[0]
            req = Request(PROJECTION, shape, observed=obs)
        else:
            w = rng.random(K)
            req = Request(BARYCENTER, shape, weights=w / w.sum())
        out.append((t, req))
    return out


def latency_summary(done):
    lat = np.array([r.latency for r in done if r.status == 0]) * 1e3
    if lat.size == 0:
        return dict(p50_ms=None, p99_ms=None, completed=0)
    return dict(p50_ms=float(np.percentile(lat, 50)), p99_ms=float(np.percentile(lat, 99)),
                mean_ms=float(lat.mean()), completed=int(lat.size),
                failed=int(sum(1 for r in done if r.status != 0)))
