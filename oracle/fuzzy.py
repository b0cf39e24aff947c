"""Fuzzy simplicial set oracle (test infrastructure): mlx_vis/_umap/umap.py:199-270.

``smooth_knn_dist`` is the per-row rho / sigma bisection of umap.py:208-236 in a
chosen float type: float32 mirrors the reference, float64 is the oracle the CUDA
kernel (which bisects in float64) is checked against.  ``fuzzy_simplicial_set``
adds the weights (umap.py:239), the symmetrisation P = A + A^T - A o A^T over the
n*k directed kNN edges (umap.py:241-262, reverse weight = first matching edge of
the reverse row) and the prune w >= max(w)/n_epochs with row-major compaction
(umap.py:265-270).
"""

from __future__ import annotations

import numpy as np


def smooth_knn_dist(knn_dists: np.ndarray, k: int, dtype=np.float64, n_iter: int = 64):
    """Returns (rho, sigma) in ``dtype``; umap.py:208-236 row by row."""
    D = np.asarray(knn_dists).astype(dtype)
    n = D.shape[0]
    t = dtype
    target = t(np.log2(k))
    rho = np.where(D > 0, D, t(np.inf)).min(axis=1)
    rho = np.maximum(rho, t(1e-8))
    lo = np.full(n, t(1e-20))
    hi = np.full(n, t(1e3))
    sigma = np.ones(n, dtype=dtype)
    ds = np.maximum(D - rho[:, None], t(0))
    tail = ds[:, 1:]
    for _ in range(n_iter):
        vals_sum = np.exp(-tail / sigma[:, None]).sum(axis=1, dtype=dtype)
        conv = np.abs(vals_sum - target) < t(1e-5)
        too_high = (vals_sum > target) & ~conv
        too_low = (vals_sum < target) & ~conv
        hi = np.where(too_high, sigma, hi)
        lo = np.where(too_low, sigma, lo)
        sigma = np.where(too_high, (lo + sigma) / t(2.0), sigma)
        sigma = np.where(too_low, np.where(hi >= t(1e3), sigma * t(2.0), (sigma + hi) / t(2.0)), sigma)
        if np.all(conv):
            break
    return rho, sigma


def edge_weights(knn_dists: np.ndarray, rho: np.ndarray, sigma: np.ndarray) -> np.ndarray:
    """umap.py:239: w = exp(-max(d - rho, 0) / max(sigma, 1e-10)), computed in the
    inputs' float type and returned as float32."""
    dt = rho.dtype
    D = np.asarray(knn_dists).astype(dt)
    ds = np.maximum(D - rho[:, None], dt.type(0))
    return np.exp(-ds / np.maximum(sigma[:, None], dt.type(1e-10))).astype(np.float32)


def symmetrize(knn_idx: np.ndarray, w: np.ndarray) -> np.ndarray:
    """umap.py:241-262 on float32 weights: w_sym = w + w_rev - w * w_rev."""
    n, k = knn_idx.shape
    rows = np.repeat(np.arange(n, dtype=np.int64), k)
    cols = knn_idx.reshape(-1).astype(np.int64)
    vals = w.reshape(-1).astype(np.float32)
    fwd = rows * n + cols
    rev = cols * n + rows
    order = np.argsort(fwd, kind="stable")
    sk = fwd[order]
    pos = np.minimum(np.searchsorted(sk, rev, side="left"), sk.size - 1)
    matched = sk[pos] == rev
    w_rev = np.where(matched, vals[order][pos], np.float32(0)).astype(np.float32)
    return ((vals + w_rev) - vals * w_rev).astype(np.float32)


def fuzzy_simplicial_set(knn_idx, knn_dists, n_epochs: int, dtype=np.float64):
    """Returns (rows int32, cols int32, vals float32) after pruning, plus (rho, sigma)."""
    knn_idx = np.asarray(knn_idx)
    n, k = knn_idx.shape
    rho, sigma = smooth_knn_dist(knn_dists, k, dtype=dtype)
    w = edge_weights(knn_dists, rho, sigma)
    w_sym = symmetrize(knn_idx, w)
    thr = np.float32(w_sym.max()) / np.float32(n_epochs)
    keep = np.nonzero(w_sym >= thr)[0]
    rows = np.repeat(np.arange(n, dtype=np.int32), k)[keep]
    cols = knn_idx.reshape(-1).astype(np.int32)[keep]
    return (rows, cols, w_sym[keep]), (rho, sigma)
