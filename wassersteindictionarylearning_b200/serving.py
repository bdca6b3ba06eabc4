"""Continuous-batching request loop for barycenter and projection requests.

Two request kinds, both against a resident dictionary of K atoms per grid shape:

* barycenter: given weights, the forward Bregman projections
  (WassersteinBarycenter::compute_barycenter, cpp/inverseWasserstein.h:115-153);
* projection: fit the K barycentric weights of one new histogram, i.e. minimise
  loss(bary(w), obs) over w on the simplex with L-BFGS — the weight half of
  compute_gradient_both (:635-673) with the atoms held fixed.

The engine keeps a device context per grid shape (LRU-bounded), admits pending
requests while the HBM bytes of the admitted requests' iterate stores fit the
budget, and sends each shape's active requests to the device as ONE batched
call (all barycenter requests of the shape in one wdl_barycenter call, one
objective evaluation for every active projection in one wdl_gradient_both
call).  Shapes run concurrently on their own contexts' streams from a thread
pool and never wait for one another: as soon as a shape's call returns, its
requests (with any that arrived meanwhile) go back to the device.  A projection
request carries a resumable L-BFGS (lbfgs.lbfgs_steps), so requests that arrive
while others are on the device join at their shape's next call and leave as
soon as their optimisation ends.
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
    form: str = ""          # "fast" (configured precision) or "fp64" (after an FP32 overflow)
    _steps: object = None
    _x: Optional[np.ndarray] = None

    @property
    def latency(self) -> float:
        return self.t_done - self.t_arrival


@dataclass(eq=False)
class _Shape:
    key: tuple              # (W, H, D, form)
    kernel: object
    atoms: np.ndarray
    active: list = field(default_factory=list)
    device_fit: bool = True  # cleared when the context's form has no device fit (fused tensor-core)


class ServingEngine:
    """Request loop.  precision: tensor-core form for 2-D shapes up to 512 per
    side (split_bf16 / tf32), FP32 operator path for 3-D shapes.

    The kernel-domain scalings of a narrow kernel grow with the iterations (for
    gamma = 2 px^2 and blob dictionaries they pass 1e60 within 50 iterations),
    beyond the FP32 range of the fast forms but inside FP64's, where the
    reference computes.  A request whose fast-form result is non-finite is
    served again from its start on the shape's FP64 context (the reference's
    arithmetic), and the shape's later requests go there directly;
    preload(calibrate=True) finds those shapes at start-up."""

    def __init__(self, K: int = 5, L: int = 50, gamma: float = 2.0, loss_type: int = 2,
                 precision: str = "split_bf16", hbm_budget: float = 8e9, max_batch: int = 64,
                 lbfgs_iterations: int = 20, max_shapes: int = 512, workers: int = 8,
                 dictionary_seed: int = 100, device: int = 0, autotune: bool = False,
                 lbfgs_epsilon: float = 1e-50, device_fit: bool = False):
        self.K, self.L, self.gamma, self.loss_type = K, L, gamma, loss_type
        self.precision = precision
        self.hbm_budget = hbm_budget
        self.max_batch = max_batch
        # regress_both's L-BFGS settings (cpp/inverseWasserstein.h:365-372): with
        # epsilon 1e-50 a projection runs its lbfgs_iterations unless the line
        # search stops it
        self.lbfgs_param = lb.LbfgsParam(max_iterations=lbfgs_iterations, epsilon=lbfgs_epsilon)
        self.max_shapes = max_shapes
        self.device = device
        # device_fit: projections on the CUDA-core forms (FP64, 3-D FP32) fit
        # their weights with the L-BFGS on the device (wdl_fit_weights_operator):
        # one call per shape batch instead of one host round trip per
        # evaluation, but a fit holds its shape until it ends, so requests that
        # arrive meanwhile no longer join the running batch (off by default:
        # the host loop served the bench mix at a higher rate)
        self.device_fit = device_fit
        self.dictionary_seed = dictionary_seed
        # a request loop keeps the default launch variants: timing variants on a
        # shape's first calls would add synchronisations to those requests
        self.autotune = autotune
        self._shapes: "OrderedDict[tuple, _Shape]" = OrderedDict()
        self.wide_shapes: set = set()  # (W, H, D) whose scalings leave the FP32 range
        self._pending: deque = deque()
        self._lock = threading.Lock()
        self._ids = itertools.count()
        self._pool = cf.ThreadPoolExecutor(max_workers=workers)
        # contexts are created and destroyed on a side pool: both can wait for the
        # device (a new context's tables are built on its stream; freeing device
        # memory synchronises), which must not hold up the request loop
        self._side = cf.ThreadPoolExecutor(max_workers=2)
        self._running: dict = {}   # shape key -> future of its call in flight
        self._creating: dict = {}  # shape key -> future of its new _Shape
        self.admitted_bytes = 0
        self.completed: list = []

    # ---- dictionary / contexts --------------------------------------------------------
    def _precision_for(self, key):
        # 2-D grids up to 512 take the tensor-core form (fused kernel up to
        # 128, axis-pass GEMMs above); the 48^3 volumes stay FP32 on the CUDA
        # cores, which is faster there (6.7 vs 7.2 ms per evaluation for K=5,
        # L=50: a 48-long axis fills little of a 128 x 64 tensor-core tile)
        W, H, D, form = key
        if form == "fp64":
            return "fp64"
        if D == 1 and W <= 512 and H <= 512 and self.precision in ("split_bf16", "tf32"):
            return self.precision
        return "fp32" if self.precision != "fp64" else "fp64"

    def dictionary(self, shape) -> np.ndarray:
        """The resident dictionary of a shape: K seeded blob atoms (fixed per
        shape, the same in both forms)."""
        geo = tuple(int(v) for v in shape[:3])
        return self._shape(self._key(geo, "fp64" if geo in self.wide_shapes else "fast")).atoms

    @staticmethod
    def _key(shape, form):
        return tuple(int(v) for v in shape[:3]) + (form,)

    def _make_shape(self, key) -> _Shape:
        W, H, D, _ = key
        prec = self._precision_for(key)
        if D > 1:
            kern = CudaGaussian3DKernel(self.gamma, W, H, D, precision=prec, device=self.device)
        else:
            kern = CudaGaussian2DKernel(self.gamma, W, H, precision=prec, device=self.device)
        if not self.autotune:
            check(lib().wdl_set_autotune(kern.ctx, 0), kern.ctx)
        seed = self.dictionary_seed + W * 7919 + H * 131 + D
        atoms = blob_histograms(self.K, W, H, D, n_blobs=(1, 3), seed=seed)
        return _Shape(key, kern, atoms)

    def _ready_shape(self, key) -> Optional[_Shape]:
        """The shape's context if it exists; otherwise its creation is started
        on the side pool (once) and None is returned until it is done."""
        s = self._shapes.get(key)
        if s is not None:
            self._shapes.move_to_end(key)
            return s
        f = self._creating.get(key)
        if f is None:
            self._creating[key] = self._side.submit(self._make_shape, key)
            return None
        if not f.done():
            return None
        del self._creating[key]
        s = f.result()
        if len(self._shapes) >= self.max_shapes:
            # evict an idle context: a fast form superseded by FP64 first, else
            # the least recently used
            idle = [k2 for k2, s2 in self._shapes.items() if not s2.active and k2 not in self._running]
            stale = [k2 for k2 in idle if k2[3] == "fast" and k2[:3] in self.wide_shapes]
            for k2 in (stale or idle)[:1]:
                self._side.submit(self._shapes.pop(k2).kernel.close)
        self._shapes[key] = s
        return s

    def _shape(self, key) -> _Shape:
        s = self._ready_shape(key)
        if s is None:
            self._creating[key].result()
            s = self._ready_shape(key)
        return s

    def _bytes(self, s: _Shape, req: Request) -> int:
        L = 2 if req.kind == BARYCENTER else self.L
        return int(lib().wdl_eval_bytes(s.kernel.ctx, 1, self.K, L))

    def _form(self, req: Request) -> str:
        if not req.form:
            geo = tuple(int(v) for v in req.shape[:3])
            req.form = "fp64" if geo in self.wide_shapes else "fast"
        return req.form

    def request_bytes(self, req: Request) -> int:
        return self._bytes(self._shape(self._key(req.shape, self._form(req))), req)

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
            return (not self._pending and not self._running and not self._creating
                    and not any(s.active for s in self._shapes.values()))

    def _admit(self):
        """Admit pending requests in arrival order while their iterate stores fit
        the budget.  A request whose shape's context is still being created
        waits, with the later requests of its shape, without holding up the
        other shapes' requests; one that does not fit (bytes or batch size)
        holds up everything behind it."""
        with self._lock:
            pending, self._pending = self._pending, deque()
        keep = deque()
        blocked = False
        waiting = set()  # shapes whose context is not ready: their later requests wait too
        for req in pending:
            if blocked:
                keep.append(req)
                continue
            key = self._key(req.shape, self._form(req))
            s = None if key in waiting else self._ready_shape(key)
            if s is None:
                waiting.add(key)
                keep.append(req)
                continue
            if not req.bytes:
                req.bytes = self._bytes(s, req)
            if req.bytes > self.hbm_budget:
                req.status = -7  # WDL_ERR_ADMISSION: can never fit
                req.t_done = time.perf_counter()
                with self._lock:
                    self.completed.append(req)
                continue
            with self._lock:
                fits = (self.admitted_bytes + req.bytes <= self.hbm_budget
                        and len(s.active) < self.max_batch)
                if fits:
                    self.admitted_bytes += req.bytes
            if not fits:
                blocked = True
                keep.append(req)
                continue
            if not req.t_admit:
                req.t_admit = time.perf_counter()
            if req.kind == PROJECTION and req._steps is None:
                x0 = np.zeros(self.K)  # uniform weights
                req._steps = lb.lbfgs_steps(x0, self.lbfgs_param)
                req._x = next(req._steps)
            with self._lock:
                s.active.append(req)
        with self._lock:
            self._pending.extendleft(reversed(keep))  # ahead of the new arrivals

    def _escalate(self, s: _Shape, req: Request):
        """The request's fast-form result left the FP32 range: it starts over on
        the shape's FP64 context, ahead of the pending requests."""
        with self._lock:
            s.active.remove(req)
            self.admitted_bytes -= req.bytes
            self.wide_shapes.add(s.key[:3])
            req.form, req.bytes, req._steps, req._x = "fp64", 0, None, None
            self._pending.appendleft(req)

    def _finish(self, s: _Shape, req: Request):
        req.t_done = time.perf_counter()
        with self._lock:
            s.active.remove(req)
            self.admitted_bytes -= req.bytes
            self.completed.append(req)

    # ---- one batched device call per shape ------------------------------------------------
    def _run_shape(self, s: _Shape):
        K, L = self.K, self.L
        ctx = s.kernel.ctx
        N = s.kernel.N
        fast = s.key[3] == "fast"
        with self._lock:
            active = list(s.active)
        bary_reqs = [r for r in active if r.kind == BARYCENTER]
        proj_reqs = [r for r in active if r.kind == PROJECTION]
        if bary_reqs:
            P = len(bary_reqs)
            w = f64(np.stack([r.weights for r in bary_reqs]))
            out = np.empty(P * N)
            rc = lib().wdl_barycenter(ctx, P, K, L, dptr(f64(s.atoms)), dptr(w), dptr(out))
            for i, r in enumerate(bary_reqs):
                res = out[i * N:(i + 1) * N]
                if rc == 0 and not np.all(np.isfinite(res)):
                    if fast:
                        self._escalate(s, r)
                        continue
                    rc_i = -5  # WDL_ERR_NONFINITE: beyond FP64's range too
                else:
                    rc_i = rc
                r.status = rc_i
                r.result = res.copy() if rc_i == 0 else None
                self._finish(s, r)
        if proj_reqs and self.device_fit and s.device_fit and self._fit_on_device(s, proj_reqs, fast):
            proj_reqs = []
        if proj_reqs:
            P = len(proj_reqs)
            # x = log-weights; lambda = normalise(exp(x)) (evaluate_both's transform, :997-1020)
            lam = np.stack([np.exp(r._x - r._x.max()) for r in proj_reqs])
            lam /= lam.sum(axis=1, keepdims=True)
            obs = f64(np.stack([r.observed for r in proj_reqs]))
            la = np.empty(P * K)
            loss = np.empty(P)
            # weights only: no atom gradient, so the dictionary recursion is skipped
            rc = lib().wdl_gradient_both(ctx, P, K, L, self.loss_type, dptr(f64(s.atoms)),
                                         dptr(f64(lam)), dptr(obs), None, dptr(la), None,
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
                    if fast:
                        self._escalate(s, r)
                        continue
                    # A trial point outside even FP64's range: report it as +inf
                    # so the line search halves the step instead of stopping.
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

    def _fit_call(self, s: _Shape, obs: np.ndarray, max_iterations: int):
        """wdl_fit_weights_operator over the rows of obs on the shape's context:
        (rc, weights [P*K], loss [P], status [P])."""
        import ctypes as C
        K, L = self.K, self.L
        P = obs.shape[0]
        obs = f64(obs.reshape(-1))
        w, f = np.empty(P * K), np.empty(P)
        st, ev = np.zeros(P, dtype=np.int32), np.zeros(P, dtype=np.int32)
        ip = C.POINTER(C.c_int)
        rc = lib().wdl_fit_weights_operator(s.kernel.ctx, P, K, L, self.loss_type, dptr(f64(s.atoms)), dptr(obs),
                                            None, max_iterations, self.lbfgs_param.epsilon, dptr(w), dptr(f),
                                            st.ctypes.data_as(ip), ev.ctypes.data_as(ip))
        return rc, w, f, st

    def _fit_on_device(self, s: _Shape, reqs, fast: bool) -> bool:
        """Fit every projection request of the batch to completion in one
        wdl_fit_weights_operator call (regress_both's L-BFGS with the atoms
        fixed, on the device, from uniform weights).  False when the shape's
        form has no device fit (the fused tensor-core form): the host L-BFGS
        serves it."""
        K = self.K
        obs = np.stack([r.observed.reshape(-1) for r in reqs])
        rc, w, f, st = self._fit_call(s, obs, self.lbfgs_param.max_iterations)
        if rc == -4:  # WDL_ERR_UNSUPPORTED
            s.device_fit = False
            return False
        for i, r in enumerate(reqs):
            if rc != 0:
                r.status = rc
                self._finish(s, r)
                continue
            if st[i] == -5:  # WDL_ERR_NONFINITE: an evaluation left the range
                if fast:
                    self._escalate(s, r)
                    continue
                r.status = -5
                self._finish(s, r)
                continue
            r.result = w[i * K:(i + 1) * K].copy()
            r.loss = float(f[i])
            r.lbfgs_status = int(st[i])
            r.status = lb.LBFGSERR_CANCELED if st[i] == lb.LBFGSERR_CANCELED else 0
            self._finish(s, r)
        return True

    def tick(self) -> int:
        """Admit what fits, collect the shape calls that have returned, then start
        one batched call for every shape with active requests and no call in
        flight.  Returns the number of calls started."""
        self._admit()
        for key, f in list(self._running.items()):
            if f.done():
                del self._running[key]
                f.result()  # a worker's exception surfaces here
        started = 0
        for s in list(self._shapes.values()):
            if s.active and s.key not in self._running:
                self._running[s.key] = self._pool.submit(self._run_shape, s)
                started += 1
        return started

    def preload(self, shapes, calibrate: bool = True):
        """Make the dictionaries of `shapes` resident before serving: their
        contexts are created concurrently on the side pool (at most max_shapes
        stay resident).  calibrate: one uniform-weight barycenter per shape in
        the fast form; a shape whose result leaves the FP32 range is served in
        FP64 from the start (its FP64 context is made resident instead)."""
        keys = [self._key(sh, "fast") for sh in shapes][: self.max_shapes]
        for key in keys:
            self._ready_shape(key)
        for key in keys:
            s = self._shape(key)
            if not calibrate:
                continue
            out = np.empty(s.kernel.N)
            w = np.full(self.K, 1.0 / self.K)
            check(lib().wdl_barycenter(s.kernel.ctx, 1, self.K, self.L, dptr(f64(s.atoms)),
                                       dptr(w), dptr(out)), s.kernel.ctx)
            if not np.all(np.isfinite(out)):
                self.wide_shapes.add(key[:3])
                self._ready_shape(key[:3] + ("fp64",))
        for key in keys:
            if key[:3] in self.wide_shapes:
                self._shape(key[:3] + ("fp64",))
                fast = self._shapes.pop(key, None)  # superseded
                if fast is not None:
                    self._side.submit(fast.kernel.close)

    def capture_graphs(self, batch_headroom: int = 2):
        """Record each resident shape's one-request projection and barycenter
        calls as CUDA graphs before serving (a projection's recorded call is the
        device fit's round where the shape has one, the host L-BFGS's
        evaluation otherwise).  A context replays a call whose
        sizes, buffers and stream it has seen twice (the first runs eagerly,
        the second is captured); those first two runs are ~1000 separate
        launches each, which a request loop on many shapes would otherwise pay
        on nearly every request.  A batch_headroom-request call first sizes the
        context's buffers, so that batches up to that size do not move them
        (which would retire the recorded graphs)."""
        K, L = self.K, self.L
        for s in list(self._shapes.values()):
            ctx, N = s.kernel.ctx, s.kernel.N
            atoms = f64(s.atoms)
            obs1 = f64(s.atoms.reshape(K, N)[0])
            if self.device_fit and s.device_fit:
                # the device fit's round (its graph does not depend on the
                # iteration limit, so two iterations record it)
                for P in (batch_headroom, 1):
                    rc = self._fit_call(s, np.tile(obs1, (P, 1)), 2)[0]
                    if rc == -4:
                        s.device_fit = False
                        break
                    check(rc, ctx)
            for P in ((batch_headroom, 1, 1) if not (self.device_fit and s.device_fit) else ()):
                lam = f64(np.full((P, K), 1.0 / K))
                obs = f64(np.tile(obs1, P))
                la, loss = np.empty(P * K), np.empty(P)
                check(lib().wdl_gradient_both(ctx, P, K, L, self.loss_type, dptr(atoms), dptr(lam),
                                              dptr(obs), None, dptr(la), None, None, dptr(loss), None), ctx)
            w, out = f64(np.full(K, 1.0 / K)), np.empty(N)
            for _ in range(2):
                check(lib().wdl_barycenter(ctx, 1, K, L, dptr(atoms), dptr(w), dptr(out)), ctx)

    def warm_up(self):
        """Serve one barycenter and one projection request per operator form
        (2-D grid up to 128, 2-D grid above 128, 3-D volume; fast and FP64) on
        small shapes and drop them: the first launch of each device kernel in a
        process pays for loading it, which a server does at start-up rather
        than inside a request."""
        shapes = [(32, 24, 1), (136, 130, 1), (12, 10, 8)]
        for form in ("fast", "fp64"):
            reqs = []
            for i, shape in enumerate(shapes):
                obs = blob_histograms(1, *shape, n_blobs=(1, 2), seed=7 + i)[0]
                reqs.append((0.0, Request(PROJECTION, shape, observed=obs, form=form)))
                reqs.append((0.0, Request(BARYCENTER, shape, weights=np.full(self.K, 1.0 / self.K),
                                          form=form)))
            self.run(reqs)
        for shape in shapes:
            self.wide_shapes.discard(shape)
            for form in ("fast", "fp64"):
                s = self._shapes.pop(self._key(shape, form), None)
                if s is not None:
                    s.kernel.close()
        self.completed = []

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
            started = self.tick()
            if not queue and self.idle():
                break
            if not started:
                # until a shape call or a context creation returns, or the next
                # request arrives (at most 1 ms)
                wait = 0.001
                if queue:
                    wait = min(wait, max(0.0, queue[0][0] - (time.perf_counter() - t0)))
                futs = list(self._running.values()) + list(self._creating.values())
                if futs:
                    cf.wait(futs, timeout=wait, return_when=cf.FIRST_COMPLETED)
                else:
                    time.sleep(wait)
            if time.perf_counter() - t0 > timeout:
                raise WdlError(-6, "serving run exceeded its timeout")
        return self.completed

    def close(self):
        self._pool.shutdown(wait=True)
        self._side.shutdown(wait=True)
        for f in self._creating.values():
            if f.exception() is None:
                f.result().kernel.close()
        self._creating.clear()
        for s in self._shapes.values():
            s.kernel.close()
        self._shapes.clear()


def poisson_requests(rate: float, n: int, seed: int = 0, K: int = 5, frac_3d: float = 0.2,
                     side_range=(64, 256), cube: int = 48, frac_projection: float = 0.5,
                     sides=None):
    """(arrival_offset, Request) pairs: Poisson arrivals at `rate` per second,
    square 2-D grids whose side is uniform in side_range (or drawn from
    `sides`), a fraction of 3-D cube^3 volumes, half projection requests
    (observed: seeded blob histograms) and half barycenter requests (weights:
    uniform on the simplex)."""
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
            s = int(rng.integers(side_range[0], side_range[1] + 1))
            shape = (s, s, 1)
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
