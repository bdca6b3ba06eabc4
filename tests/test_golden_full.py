"""CPU: the full-grid fixtures (tests/golden/full_*.npz) are usable on any host.

They store no inputs: the GPU tests regenerate them from the recorded seeds.
This checks, without a GPU, that the regeneration reproduces the reference
run's inputs (the stored input statistics) and that each stored sample is
consistent with its whole-array statistics."""
import numpy as np
import pytest

from conftest import golden


def _stats(*arrays):
    return np.array([v for a in arrays for v in (float(np.sum(a)), float(np.sum(np.asarray(a) ** 2)),
                                                  float(np.max(a)), float(np.min(a)))])


def _inputs(name, f):
    from wassersteindictionarylearning_b200.synthetic import blob_histograms, init_atoms, init_weights
    if name.startswith("full_logconv"):
        W, H = int(f["W"]), int(f["H"])
        rng = np.random.Generator(np.random.PCG64(int(f["seed"])))
        return (np.log(rng.random(W * H)) * 3.0,)
    a, b, c = (int(v) for v in f["seeds"])
    W, H, K = int(f["W"]), int(f["H"]), int(f["K"])
    D = int(f["D"]) if "D" in f else 1
    P = int(f["P"]) if "P" in f else 1
    std = (0.05, 0.12) if D > 1 else (0.01, 0.04)
    obs = blob_histograms(P, W, H, D, n_blobs=(1, 3), std_frac=std, seed=a)
    if P == 1:
        obs = obs[0]
    w = init_weights(P, K, seed=c)
    return obs, init_atoms(K, W * H * D, seed=b), (w[0] if P == 1 else w)


@pytest.mark.parametrize("name,f", golden("full_*"))
def test_full_fixture_inputs_regenerate(name, f):
    assert np.allclose(_stats(*_inputs(name, f)), f["in_stats"], rtol=1e-12, atol=0)


@pytest.mark.parametrize("name,f", golden("full_*"))
def test_full_fixture_samples_consistent(name, f):
    prefixes = {k[: -len("_sample")] for k in f if k.endswith("_sample")}
    assert prefixes
    for p in prefixes:
        s = f[p + "_sample"]
        assert s.size == -(-int(f[p + "_n"]) // int(f[p + "_stride"]))
        assert np.max(np.abs(s)) <= float(f[p + "_absmax"])
        assert np.sum(np.abs(s)) <= float(f[p + "_abssum"])
