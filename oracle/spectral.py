"""Spectral initialisation oracle (test infrastructure): mlx_vis/_umap/umap.py:298-357.

The reference draws the start block V (n x (c+1)) from MLX's RNG, which cannot be
reproduced without MLX, so V0 is an argument (the golden fixture stores the draw
of the NumPy-backed shim).  Everything else follows the reference: degree
scatter-add, D^-1/2 W D^-1/2, 100 power iterations each followed by modified
Gram-Schmidt (norm = sqrt(|v|^2 + 1e-10)), columns 1..c, scale by 10/max|e|,
N(0, 1e-4) noise from ``np.random.RandomState(random_state or 42)`` and a
per-column min-max rescale to [0, 10].
"""

from __future__ import annotations

import numpy as np


def power_iteration(rows, cols, vals, n: int, V0: np.ndarray, n_iter: int = 100,
                    dtype=np.float64) -> np.ndarray:
    """umap.py:305-337 in ``dtype``; returns V (n x (c+1)) after the last MGS."""
    rows = np.asarray(rows, dtype=np.int64)
    cols = np.asarray(cols, dtype=np.int64)
    w = np.asarray(vals).astype(dtype)
    deg = np.zeros(n, dtype=dtype)
    np.add.at(deg, rows, w)
    deg = np.maximum(deg, dtype(1e-10))
    dis = dtype(1.0) / np.sqrt(deg)
    wn = w * dis[rows] * dis[cols]
    V = np.asarray(V0).astype(dtype).copy()
    kk = V.shape[1]
    for _ in range(n_iter):
        out = np.zeros_like(V)
        np.add.at(out, rows, wn[:, None] * V[cols])
        V = out
        for j in range(kk):
            for i in range(j):
                V[:, j] -= np.sum(V[:, j] * V[:, i]) * V[:, i]
            V[:, j] *= dtype(1.0) / np.sqrt(np.sum(V[:, j] * V[:, j]) + dtype(1e-10))
    return V


def rescale(embedding: np.ndarray, random_state) -> np.ndarray:
    """umap.py:343-348 (float32, NumPy RandomState noise)."""
    e = np.asarray(embedding, dtype=np.float32)
    rng = np.random.RandomState(random_state or 42)
    expansion = 10.0 / np.max(np.abs(e))
    e = (e * expansion).astype(np.float32)
    e += rng.normal(scale=0.0001, size=e.shape).astype(np.float32)
    return 10.0 * (e - e.min(axis=0)) / (e.max(axis=0) - e.min(axis=0) + 1e-10)


def spectral_init(rows, cols, vals, n: int, V0: np.ndarray, random_state, n_iter: int = 100,
                  dtype=np.float64) -> np.ndarray:
    V = power_iteration(rows, cols, vals, n, V0, n_iter=n_iter, dtype=dtype)
    return rescale(V[:, 1:].astype(np.float32), random_state)
