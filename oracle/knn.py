"""Brute-force kNN oracles (test infrastructure).

``knn_expanded_f32`` restates the reference's brute path, mlx_vis/_knn.py:47-88:
row chunks of ``min(n, max(1000, 5e8 // (4 n)))``, D = max(|x|^2 + |y|^2 - 2 x.y, 0)
in float32, self distance + 1e30, full-row argsort, first k, then sqrt.

``knn_exact_f64`` is the float64 ground truth (direct differences), ties broken
by index.
"""

from __future__ import annotations

import numpy as np


def knn_expanded_f32(X: np.ndarray, k: int, return_euclidean: bool = True):
    """mlx_vis/_knn.py:47-88 in NumPy float32 (stable argsort for ties)."""
    X = np.asarray(X, dtype=np.float32)
    n = X.shape[0]
    sq = np.sum(X * X, axis=1, dtype=np.float32)
    chunk = min(n, max(1000, 500_000_000 // (n * 4)))
    idx = np.zeros((n, k), dtype=np.int32)
    d2 = np.zeros((n, k), dtype=np.float32)
    for s in range(0, n, chunk):
        e = min(s + chunk, n)
        D = np.maximum(sq[s:e, None] + sq[None, :] - np.float32(2.0) * (X[s:e] @ X.T), np.float32(0))
        D[np.arange(e - s), np.arange(s, e)] += np.float32(1e30)
        o = np.argsort(D, axis=1, kind="stable")[:, :k]
        idx[s:e] = o
        d2[s:e] = np.take_along_axis(D, o, axis=1)
    if return_euclidean:
        return idx, np.sqrt(np.maximum(d2, 0)).astype(np.float32)
    return idx, d2


def sqdist_f64(X: np.ndarray, rows: np.ndarray, cols: np.ndarray) -> np.ndarray:
    """Exact float64 squared distances between X[rows[i]] and X[cols[i, j]]."""
    X64 = np.asarray(X, dtype=np.float64)
    diff = X64[np.asarray(cols)] - X64[np.asarray(rows)][:, None, :]
    return np.einsum("ijd,ijd->ij", diff, diff)


def knn_exact_f64(X: np.ndarray, k: int, chunk: int = 512):
    """Exact kNN in float64: returns (idx int32 (n,k), d2 float64 (n,k)), ascending,
    self excluded, equal distances ordered by index."""
    X64 = np.asarray(X, dtype=np.float64)
    n = X64.shape[0]
    sq = np.einsum("ij,ij->i", X64, X64)
    idx = np.zeros((n, k), dtype=np.int32)
    d2 = np.zeros((n, k), dtype=np.float64)
    for s in range(0, n, chunk):
        e = min(s + chunk, n)
        D = sq[s:e, None] + sq[None, :] - 2.0 * (X64[s:e] @ X64.T)
        D[np.arange(e - s), np.arange(s, e)] = np.inf
        # candidates by the expanded form, then exact re-evaluation by differences
        m = min(n - 1, k + 32)
        cand = np.argpartition(D, m - 1, axis=1)[:, :m]
        diff = X64[cand] - X64[s:e, None, :]
        dd = np.einsum("ijd,ijd->ij", diff, diff)
        order = np.lexsort((cand, dd), axis=1)[:, :k]
        idx[s:e] = np.take_along_axis(cand, order, axis=1)
        d2[s:e] = np.take_along_axis(dd, order, axis=1)
    return idx, d2
