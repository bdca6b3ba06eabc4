"""GPU: the continuous-batching serving loop.

Each request's result is the same served alone and served inside a mixed
stream (other shapes and kinds arriving while it runs): bitwise in FP64 (the
FP64 path has no atomics), within tolerance on the split-BF16 path (whose
cross-atom sums use float atomics).  Admission by iterate-store bytes: a request
that can never fit is refused, the rest still complete; barycenter results match
the oracle."""
import numpy as np
import pytest

from conftest import rel

pytestmark = pytest.mark.gpu


def _stream(n, seed, sides=(32, 48, 64), frac_3d=0.2, cube=12, rate=400.0):
    from wassersteindictionarylearning_b200.serving import poisson_requests
    return poisson_requests(rate, n, seed=seed, K=3, frac_3d=frac_3d, sides=sides, cube=cube)


def _engine(precision, gamma=2.0, **kw):
    from wassersteindictionarylearning_b200.serving import ServingEngine
    return ServingEngine(K=3, L=12, gamma=gamma, loss_type=2, precision=precision,
                         lbfgs_iterations=8, **kw)


@pytest.mark.parametrize("precision,tol_b,tol_w", [("fp64", 0.0, 0.0), ("split_bf16", 1e-5, 2e-3)])
def test_alone_equals_mixed(precision, tol_b, tol_w):
    import copy
    arr = _stream(16, seed=3)
    eng = _engine(precision)
    done = {r.rid: r for r in eng.run(copy.deepcopy(arr))}
    eng.close()
    mixed = sorted(done.values(), key=lambda r: r.rid)
    assert len(mixed) == 16 and all(r.status == 0 for r in mixed)
    for i, (_, req) in enumerate(arr):
        eng1 = _engine(precision)
        alone = eng1.run([(0.0, copy.deepcopy(req))])[0]
        eng1.close()
        m = mixed[i]
        assert m.kind == alone.kind and m.shape == alone.shape
        if tol_b == 0.0:
            assert np.array_equal(m.result, alone.result), (m.kind, m.shape)
        elif m.kind == "barycenter":
            assert rel(m.result, alone.result) < tol_b
        else:
            assert np.max(np.abs(m.result - alone.result)) < tol_w


def test_barycenter_requests_match_oracle(oracle):
    from wassersteindictionarylearning_b200.serving import BARYCENTER, Request
    eng = _engine("fp64")
    reqs = []
    for i, shape in enumerate([(20, 16, 1), (20, 16, 1), (9, 8, 7)]):
        w = np.array([0.2, 0.5, 0.3]) + 0.1 * i
        reqs.append((0.0, Request(BARYCENTER, shape, weights=w / w.sum())))
    done = sorted(eng.run(reqs), key=lambda r: r.rid)
    for r in done:
        W, H, D = r.shape
        ref = oracle.barycenter(W, H, D, 2.0, 3, 12, eng.dictionary(r.shape), r.weights)
        assert rel(r.result, ref) < 1e-10
    eng.close()


def test_admission_by_bytes():
    from wassersteindictionarylearning_b200.serving import PROJECTION, Request
    from wassersteindictionarylearning_b200.synthetic import blob_histograms
    big = Request(PROJECTION, (64, 64, 1), observed=blob_histograms(1, 64, 64, seed=1)[0])
    small = [Request(PROJECTION, (32, 32, 1), observed=blob_histograms(1, 32, 32, seed=2 + i)[0])
             for i in range(3)]
    # gamma 8: the FP32 scalings stay in range, so no request moves to FP64
    probe = _engine("fp32", gamma=8.0)
    b_small, b_big = probe.request_bytes(small[0]), probe.request_bytes(big)
    probe.close()
    assert b_big > 1.6 * b_small
    eng = _engine("fp32", gamma=8.0, hbm_budget=1.5 * b_small)  # room for one small request at a time
    done = eng.run([(0.0, big)] + [(0.0, s) for s in small])
    st = {r.rid: r.status for r in done}
    assert st[0] == -7                       # WDL_ERR_ADMISSION: never fits
    assert all(st[i] == 0 for i in (1, 2, 3))  # served one after another
    order = [r.rid for r in done if r.status == 0]
    assert order == [1, 2, 3]
    assert eng.admitted_bytes == 0 and not eng.wide_shapes
    eng.close()


def test_fp32_overflow_is_served_in_fp64():
    """Blob dictionary, gamma 2, L 50 on a 64 x 64 grid: the kernel-domain
    scalings pass 1e60, beyond FP32 and inside FP64.  The split-BF16 engine's
    requests start over on the shape's FP64 context, so they return exactly
    what an FP64 engine returns; start-up calibration finds the shape too."""
    import copy

    from wassersteindictionarylearning_b200.serving import (BARYCENTER, PROJECTION, Request,
                                                            ServingEngine)
    from wassersteindictionarylearning_b200.synthetic import blob_histograms
    shape = (64, 64, 1)
    reqs = [(0.0, Request(PROJECTION, shape, observed=blob_histograms(1, 64, 64, seed=9)[0])),
            (0.0, Request(BARYCENTER, shape, weights=np.array([0.1, 0.2, 0.3, 0.25, 0.15])))]

    def mk(precision):
        return ServingEngine(K=5, L=50, gamma=2.0, loss_type=2, precision=precision,
                             lbfgs_iterations=4)
    eng, ref = mk("split_bf16"), mk("fp64")
    got = sorted(eng.run(copy.deepcopy(reqs)), key=lambda r: r.rid)
    want = sorted(ref.run(copy.deepcopy(reqs)), key=lambda r: r.rid)
    assert shape in eng.wide_shapes
    for g, w in zip(got, want):
        assert g.status == 0 and g.form == "fp64" and np.all(np.isfinite(g.result))
        assert np.array_equal(g.result, w.result), g.kind
    eng.close()
    ref.close()
    cal = mk("split_bf16")
    cal.preload([shape])
    assert shape in cal.wide_shapes
    cal.close()


def test_recorded_graphs_serve_the_same_results():
    """capture_graphs() records every resident shape's one-request projection
    and barycenter calls as CUDA graphs; requests served afterwards (replays)
    return bitwise what an engine without recorded graphs returns (FP64)."""
    import copy
    arr = _stream(10, seed=5, frac_3d=0.3)
    shapes = sorted({req.shape for _, req in arr})
    results = []
    for record in (False, True):
        eng = _engine("fp64")
        eng.preload(shapes, calibrate=False)
        if record:
            eng.capture_graphs()
        done = sorted(eng.run(copy.deepcopy(arr)), key=lambda r: r.rid)
        eng.close()
        assert len(done) == 10 and all(r.status == 0 for r in done)
        results.append(done)
    for a, b in zip(*results):
        assert a.kind == b.kind and a.shape == b.shape
        assert np.array_equal(a.result, b.result), (a.kind, a.shape)


def test_device_fit_serves_the_host_fits():
    """With device_fit the FP64 projections run wdl_fit_weights_operator (the
    L-BFGS on the device) and return the host L-BFGS's weights."""
    import copy
    arr = _stream(8, seed=9, frac_3d=0.3)
    outs = []
    for device_fit in (False, True):
        eng = _engine("fp64", device_fit=device_fit)
        done = sorted(eng.run(copy.deepcopy(arr)), key=lambda r: r.rid)
        eng.close()
        assert len(done) == 8 and all(r.status == 0 for r in done)
        outs.append(done)
    for a, b in zip(*outs):
        assert a.kind == b.kind and a.shape == b.shape
        if a.kind == "projection":
            assert a.lbfgs_status == b.lbfgs_status
            assert np.max(np.abs(a.result - b.result)) < 1e-8
        else:
            assert np.array_equal(a.result, b.result)
