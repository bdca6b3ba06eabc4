"""Seeded synthetic inputs with the shapes of the reference's use (no dataset ships).

Histograms are mixtures of anisotropic Gaussian blobs evaluated at pixel
centres, floored at 1e-6 and normalised to sum 1 — the stand-in for the
images the reference loads with ``load_img_to_pdf_gamma_correction``
(cpp/histogramIO.h:287-312).  Atom and weight initialisation follows
cpp/main_dictionary_learning.cpp:122-153 (atoms uniform, here with a small
seeded perturbation; weights uniform in [0, 1] then normalised).

Layouts match the reference: an image is row-major with x fastest
(index ``y*W + x``; 3-D ``z*W*H + y*W + x``), histograms are stacked with
stride N, and the optimisation vector is ``[P*K weights, K*N atoms]``.
"""
from __future__ import annotations

import numpy as np


def blob_histograms(P: int, W: int, H: int, D: int = 1, n_blobs=(1, 3), std_frac=(0.03, 0.12),
                    seed: int = 0, floor: float = 1e-6) -> np.ndarray:
    """P histograms of size N = W*H*D as a (P, N) float64 array, each summing to 1."""
    rng = np.random.Generator(np.random.PCG64(seed))
    side = np.array([W, H, D][: 3 if D > 1 else 2], dtype=np.float64)
    dims = len(side)
    axes = [np.arange(n) + 0.5 for n in ([W, H, D] if D > 1 else [W, H])]
    grid = np.stack(np.meshgrid(*axes, indexing="ij"), axis=-1)  # (W, H[, D], dims)
    out = np.empty((P, W * H * D), dtype=np.float64)
    for p in range(P):
        nb = int(rng.integers(n_blobs[0], n_blobs[1] + 1))
        mix = rng.dirichlet(np.ones(nb))
        dens = np.zeros(grid.shape[:-1])
        for b in range(nb):
            centre = rng.uniform(0.2, 0.8, size=dims) * side
            std = rng.uniform(std_frac[0], std_frac[1], size=dims) * side
            if dims == 2:
                t = rng.uniform(0.0, np.pi)
                R = np.array([[np.cos(t), -np.sin(t)], [np.sin(t), np.cos(t)]])
            else:  # random rotation from the QR of a Gaussian matrix
                q, r = np.linalg.qr(rng.standard_normal((3, 3)))
                R = q * np.sign(np.diag(r))
            cov = R @ np.diag(std ** 2) @ R.T
            icov = np.linalg.inv(cov)
            d = grid - centre
            m = np.einsum("...i,ij,...j->...", d, icov, d)
            g = np.exp(-0.5 * m) / np.sqrt((2 * np.pi) ** dims * np.linalg.det(cov))
            dens += mix[b] * g
        # grid is indexed (x, y[, z]); the reference layout is z-major, x fastest.
        img = np.transpose(dens, tuple(range(dims))[::-1]).reshape(-1)
        img = img + floor
        out[p] = img / img.sum()
    return out


def init_atoms(K: int, N: int, seed: int = 1, noise: float = 0.1) -> np.ndarray:
    """(K, N) atoms, 1 + noise*U[0,1) normalised to sum 1."""
    rng = np.random.Generator(np.random.PCG64(seed))
    a = 1.0 + noise * rng.random((K, N))
    return a / a.sum(axis=1, keepdims=True)


def init_weights(P: int, K: int, seed: int = 2) -> np.ndarray:
    """(P, K) barycentric weights, U[0,1] normalised per histogram."""
    rng = np.random.Generator(np.random.PCG64(seed))
    w = rng.random((P, K))
    return w / w.sum(axis=1, keepdims=True)


def scale_dictionary(N: int, P: int, factor: float = 100.0) -> float:
    """scaleDictionary = (N/P)/scaleDictFactor (cpp/main_dictionary_learning.cpp:138)."""
    return (N / float(P)) / factor


def to_variables(weights: np.ndarray, atoms: np.ndarray, scale_dic: float) -> np.ndarray:
    """Original-domain (weights, atoms) -> the L-BFGS vector x of regress_both
    (cpp/inverseWasserstein.h:389-401): log(weights)*scale, log(atoms)."""
    return np.concatenate([np.log(weights.reshape(-1)) * scale_dic, np.log(atoms.reshape(-1))])


# Named workloads (sizes as in the benchmark configurations).
WORKLOADS = {
    "dict64": dict(P=16, W=64, H=64, D=1, K=4, L=25, gamma=2.0, loss=2, n_blobs=(1, 3),
                   std_frac=(0.03, 0.12), lbfgs_iters=20),
    "batched128": dict(P=64, W=128, H=128, D=1, K=5, L=100, gamma=1.0, loss=4, n_blobs=(2, 5),
                       std_frac=(0.03, 0.12), lbfgs_iters=50),
    "log256": dict(P=32, W=256, H=256, D=1, K=8, L=200, gamma=0.5, loss=1, n_blobs=(1, 3),
                   std_frac=(0.01, 0.04), lbfgs_iters=30),
}


def make_problem(name: str = None, seed: int = 0, **overrides):
    """Histograms, atoms, weights and scale for a named workload (overridable)."""
    cfg = dict(WORKLOADS[name]) if name else {}
    cfg.update(overrides)
    P, W, H, D, K = cfg["P"], cfg["W"], cfg["H"], cfg.get("D", 1), cfg["K"]
    N = W * H * D
    obs = blob_histograms(P, W, H, D, n_blobs=cfg.get("n_blobs", (1, 3)),
                          std_frac=cfg.get("std_frac", (0.03, 0.12)), seed=seed)
    atoms = init_atoms(K, N, seed=seed + 1)
    weights = init_weights(P, K, seed=seed + 2)
    cfg["scale_dic"] = scale_dictionary(N, P)
    return cfg, obs, atoms, weights
