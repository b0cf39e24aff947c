"""PCA preprocessing oracle (test infrastructure): mlx_vis/_umap/umap.py:92-113.

mean over rows, X - mean, covariance (X - mean)^T (X - mean) / (n - 1), eigh
(ascending eigenvalues), the last pca_dim eigenvectors in reverse order as the
projection, (X - mean) @ projection.  Everything in float64; eigenvector signs
are whatever LAPACK returns, so comparisons are per column up to sign.
"""

from __future__ import annotations

import numpy as np


def pca(X: np.ndarray, pca_dim: int):
    """Returns (X_pca float64 (n, pca_dim), eigenvalues ascending, projection (d, pca_dim))."""
    X = np.asarray(X, dtype=np.float64)
    n = X.shape[0]
    mean = X.mean(axis=0)
    Xc = X - mean
    cov = (Xc.T @ Xc) / (n - 1)
    w, v = np.linalg.eigh(cov)
    proj = v[:, -pca_dim:][:, ::-1]
    return Xc @ proj, w, proj


def align_signs(A: np.ndarray, B: np.ndarray) -> np.ndarray:
    """B with each column's sign flipped where that brings it closer to A's column."""
    s = np.sign(np.sum(A * B, axis=0))
    s[s == 0] = 1.0
    return B * s
