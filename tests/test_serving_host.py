"""CPU: the serving loop's host logic, on a stand-in for the device library.

The request loop (admission by bytes, one batched call per shape, shapes
running independently, contexts created off the loop, FP64 re-serving of
requests whose fast-form results come back non-finite, start-up calibration)
is plain Python.  Here the library is replaced by a numpy model with the same
calling convention: barycenter = weights @ atoms, quadratic loss and its weight
gradient; a "fast" context of a shape listed as out of range returns NaN, as
the FP32 forms do when the kernel-domain scalings leave their range.  The GPU
tests run the same loop on the real kernels."""
import threading
import time

import numpy as np
import pytest

from wassersteindictionarylearning_b200 import serving


class _Ctx:
    def __init__(self, shape, precision):
        self.shape, self.precision = shape, precision
        self.N = int(np.prod(shape))


class _Kernel:
    def __init__(self, gamma, W, H, D=1, precision="fp32", device=0):
        self.ctx = _Ctx((W, H, D), precision)
        self.N = self.ctx.N

    def close(self):
        pass


class _FakeLib:
    """numpy model of wdl_barycenter / wdl_gradient_both (weights only)."""

    def __init__(self, out_of_range=(), slow=(), delay=0.0, device_fit=False):
        self.out_of_range, self.slow, self.delay = set(out_of_range), set(slow), delay
        self.device_fit = device_fit
        self.calls = []
        self.lock = threading.Lock()

    def _view(self, p, n):
        return np.ctypeslib.as_array(p, shape=(n,))

    def _bad(self, ctx):
        return ctx.precision != "fp64" and ctx.shape in self.out_of_range

    def _log(self, ctx, kind, P):
        with self.lock:
            self.calls.append((ctx.shape, ctx.precision, kind, P, time.perf_counter()))
        if ctx.shape in self.slow:
            time.sleep(self.delay)

    def wdl_set_autotune(self, ctx, on):
        return 0

    def wdl_eval_bytes(self, ctx, P, K, L):
        return ctx.N * K * L * (8 if ctx.precision == "fp64" else 4) * P

    def wdl_barycenter(self, ctx, P, K, L, atoms, w, out):
        self._log(ctx, "bary", P)
        N = ctx.N
        a = self._view(atoms, K * N).reshape(K, N)
        lam = self._view(w, P * K).reshape(P, K)
        o = self._view(out, P * N)
        # row by row, so that a request's result does not depend on its batch
        o[:] = np.nan if self._bad(ctx) else np.concatenate([l @ a for l in lam])
        return 0

    def wdl_gradient_both(self, ctx, P, K, L, loss_type, atoms, w, obs, b_init, la, dic, bary, loss,
                          b_last):
        assert dic is None  # projections ask for the weight gradient alone
        self._log(ctx, "grad", P)
        N = ctx.N
        a = self._view(atoms, K * N).reshape(K, N)
        lam = self._view(w, P * K).reshape(P, K)
        ob = self._view(obs, P * N).reshape(P, N)
        d = np.stack([l @ a for l in lam]) - ob
        g = np.stack([2.0 * (a @ di) for di in d])
        f = np.array([di @ di for di in d])
        if self._bad(ctx):
            g[:], f[:] = np.nan, np.nan
        self._view(la, P * K)[:] = g.reshape(-1)
        self._view(loss, P)[:] = f
        return 0

    def wdl_fit_weights_operator(self, ctx, P, K, L, loss_type, atoms, obs, x0, iters, eps, w, loss,
                                 status, evals):
        """-4 (unsupported: the fused tensor-core answer) unless device_fit; then
        a whole fit in one call: the least-squares weights of the numpy model,
        or status -5 (non-finite) where the model leaves the range."""
        if not self.device_fit:
            return -4
        self._log(ctx, "fit", P)
        N = ctx.N
        a = self._view(atoms, K * N).reshape(K, N)
        ob = self._view(obs, P * N).reshape(P, N)
        wv, fv = self._view(w, P * K).reshape(P, K), self._view(loss, P)
        st = np.ctypeslib.as_array(status, shape=(P,))
        ev = np.ctypeslib.as_array(evals, shape=(P,))
        for p in range(P):
            x = np.clip(np.linalg.lstsq(a.T, ob[p], rcond=None)[0], 0, None) + 1e-12
            wv[p] = x / x.sum()
            d = wv[p] @ a - ob[p]
            fv[p] = d @ d
            st[p] = -5 if self._bad(ctx) else 0
            ev[p] = iters + 1
        return 0


@pytest.fixture
def fake(monkeypatch):
    def install(**kw):
        lib = _FakeLib(**kw)
        monkeypatch.setattr(serving, "lib", lambda: lib)
        monkeypatch.setattr(serving, "check", lambda rc, ctx=None: None)
        monkeypatch.setattr(serving, "CudaGaussian2DKernel",
                            lambda g, W, H, precision, device: _Kernel(g, W, H, 1, precision, device))
        monkeypatch.setattr(serving, "CudaGaussian3DKernel", _Kernel)
        return lib
    return install


def _requests(shapes, seed=0, K=3):
    rng = np.random.default_rng(seed)
    out = []
    for i, sh in enumerate(shapes):
        N = int(np.prod(sh))
        if i % 2 == 0:
            obs = rng.random(N)
            out.append((0.0, serving.Request(serving.PROJECTION, sh, observed=obs / obs.sum())))
        else:
            w = rng.random(K)
            out.append((0.0, serving.Request(serving.BARYCENTER, sh, weights=w / w.sum())))
    return out


def _engine(**kw):
    return serving.ServingEngine(K=3, L=4, gamma=2.0, loss_type=2, precision="split_bf16",
                                 lbfgs_iterations=6, **kw)


def test_out_of_range_requests_are_served_in_fp64(fake):
    import copy
    shapes = [(8, 8, 1), (9, 9, 1), (8, 8, 1), (9, 9, 1), (4, 4, 3), (9, 9, 1)]
    reqs = _requests(shapes)
    lib = fake(out_of_range={(9, 9, 1)})
    eng = _engine()
    got = {r.rid: r for r in eng.run(copy.deepcopy(reqs))}
    eng.close()
    assert len(got) == len(shapes) and all(r.status == 0 for r in got.values())
    assert eng.wide_shapes == {(9, 9, 1)}
    for rid, r in got.items():
        assert r.form == ("fp64" if tuple(r.shape) == (9, 9, 1) else "fast")
        assert np.all(np.isfinite(r.result))
    # the re-served requests equal an FP64 engine's (they started over from scratch)
    fake(out_of_range=())
    ref = serving.ServingEngine(K=3, L=4, gamma=2.0, loss_type=2, precision="fp64",
                                lbfgs_iterations=6)
    want = {r.rid: r for r in ref.run(copy.deepcopy(reqs))}
    ref.close()
    for rid in got:
        assert np.array_equal(got[rid].result, want[rid].result)
    # every fast-form call of the wide shape happened before it was marked wide
    assert any(c[0] == (9, 9, 1) and c[1] == "fp64" for c in lib.calls)


def test_calibration_finds_out_of_range_shapes(fake):
    fake(out_of_range={(9, 9, 1)})
    eng = _engine()
    eng.preload([(8, 8, 1), (9, 9, 1), (4, 4, 3)])
    assert eng.wide_shapes == {(9, 9, 1)}
    assert (9, 9, 1, "fp64") in eng._shapes and (9, 9, 1, "fast") not in eng._shapes
    eng.close()


def test_shapes_do_not_wait_for_each_other(fake):
    """A slow shape's calls must not hold up another shape's requests."""
    lib = fake(slow={(12, 12, 1)}, delay=0.05)
    reqs = _requests([(12, 12, 1), (12, 12, 1), (8, 8, 1), (8, 8, 1)], seed=3)
    eng = _engine()
    eng.preload([(12, 12, 1), (8, 8, 1)])
    lib.calls.clear()  # the start-up calibration's calls
    done = {r.rid: r for r in eng.run(reqs)}
    eng.close()
    assert all(r.status == 0 for r in done.values())
    fast_done = max(r.t_done for r in done.values() if tuple(r.shape) == (8, 8, 1))
    slow_done = max(r.t_done for r in done.values() if tuple(r.shape) == (12, 12, 1))
    assert fast_done < slow_done
    # the fast shape made several calls while the slow one was in its first ones
    slow_first = min(c[4] for c in lib.calls if c[0] == (12, 12, 1))
    fast_calls = [c for c in lib.calls if c[0] == (8, 8, 1) and c[4] < slow_first + 0.05]
    assert len(fast_calls) >= 2


def test_admission_holds_requests_beyond_the_budget(fake):
    fake()
    reqs = _requests([(8, 8, 1), (8, 8, 1), (8, 8, 1)] * 2, seed=5)
    reqs = [(t, r) for t, r in reqs if r.kind == serving.PROJECTION]
    probe = _engine()
    b = probe.request_bytes(reqs[0][1])
    probe.close()
    eng = _engine(hbm_budget=1.5 * b)  # one projection at a time
    peak = []
    orig = eng._admit

    def admit():
        orig()
        peak.append(eng.admitted_bytes)
    eng._admit = admit
    done = eng.run(reqs)
    eng.close()
    assert len(done) == len(reqs) and all(r.status == 0 for r in done)
    assert max(peak) <= 1.5 * b and eng.admitted_bytes == 0
    assert [r.rid for r in done] == sorted(r.rid for r in done)  # served in arrival order


def test_device_fits_serve_projections_in_one_call(fake):
    """With the device fit available, a shape batch's projections finish in one
    wdl_fit_weights_operator call; a fast-form fit that leaves the range starts
    over in FP64 and is fitted there."""
    lib = fake(out_of_range={(6, 5, 1)}, device_fit=True)
    eng = _engine(device_fit=True)
    arr = [(0.0, r) for _, r in _requests([(6, 5, 1), (4, 4, 1), (6, 5, 1), (3, 3, 2)], seed=4)]
    done = sorted(eng.run(arr), key=lambda r: r.rid)
    eng.close()
    assert len(done) == 4 and all(r.status == 0 for r in done)
    fits = [c for c in lib.calls if c[2] == "fit"]
    assert not [c for c in lib.calls if c[2] == "grad"]  # no host L-BFGS evaluations
    assert ((6, 5, 1), "fp64") in {(c[0], c[1]) for c in fits}  # the escalated projection
    for r in done:
        if r.kind == serving.PROJECTION:
            assert r.result.shape == (3,) and abs(r.result.sum() - 1) < 1e-12 and r.lbfgs_status == 0
