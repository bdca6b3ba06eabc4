"""CPU: how batch.fit_weights routes weight fits between the two domains.

Problems whose side fits the tensor-core tile go to the kernel-domain device
fit, one call per gamma; a problem whose kernel-domain evaluation overflowed
(status WDL_FIT_OVERFLOW) is fitted again from its start in the log domain, and
the evaluations it already spent are added to its count; problems above the
tile go to the log domain directly, one call per gamma.  The device calls are
replaced here by a stand-in that records them; the GPU tests run the real
ones."""
import numpy as np

from wassersteindictionarylearning_b200 import batch
from wassersteindictionarylearning_b200._lib import WDL_FIT_OVERFLOW


class _Kern:
    def __init__(self, gamma, W, H, precision="fp32", device=0):
        self.gamma, self.side, self.log = gamma, (W, H), False

    def close(self):
        pass


class _LogKern(_Kern):
    def __init__(self, *a, **kw):
        super().__init__(*a, **kw)
        self.log = True


def test_fit_weights_routes_by_side_and_overflow(monkeypatch):
    calls = []

    def fake_fit_device(kern, problems, iters, eps, log_domain=False):
        assert log_domain == kern.log
        calls.append((kern.gamma, kern.log, [p["id"] for p in problems]))
        out = []
        for p in problems:
            K = p["K"]
            w = np.full((1, K), 1.0 / K)
            if not log_domain and p["overflows"]:
                st, ev = WDL_FIT_OVERFLOW, 3
            else:
                st, ev = -997, 10
            out.append((w, np.array([0.5]), np.array([st], dtype=np.int32),
                        np.array([ev], dtype=np.int32)))
        return out

    monkeypatch.setattr(batch, "fit_device", fake_fit_device)
    monkeypatch.setattr(batch, "CudaGaussian2DKernel", _Kern)
    monkeypatch.setattr(batch, "CudaLogSignArrayGaussian2DKernel", _LogKern)
    spec = [(32, 1.0, False), (64, 1.0, True), (192, 1.0, False), (48, 2.0, False),
            (160, 2.0, False), (128, 2.0, True)]
    probs = [dict(id=i, W=s, H=s, K=3, L=5, gamma=g, overflows=o, loss_type=2,
                  atoms=np.zeros(3 * s * s), observed=np.zeros(s * s))
             for i, (s, g, o) in enumerate(spec)]
    res = batch.fit_weights(probs, lbfgs_iterations=4)
    kernel_calls = {g: ids for g, log, ids in calls if not log}
    log_calls = {g: sorted(ids) for g, log, ids in calls if log}
    assert kernel_calls == {1.0: [0, 1], 2.0: [3, 5]}       # sides <= 128, per gamma
    assert log_calls == {1.0: [1, 2], 2.0: [4, 5]}          # overflowed + above the tile
    for i, (side, g, o) in enumerate(spec):
        w, f, st, ev, dom = res[i]
        log = o or side > 128
        assert dom == ("log" if log else "kernel")
        assert ev == (10 + 3 if o else 10)                  # spent evaluations carried over
        assert abs(w.sum() - 1.0) < 1e-12
