"""Layout optimisation oracle (test infrastructure): mlx_vis/_umap/umap.py:359-449.

* ``epochs_per_sample`` / ``active_sets`` restate the host schedule of
  umap.py:398-414 exactly, in float32 as NumPy 2 evaluates it there.
* ``sgd_epoch`` restates ``_sgd_step`` (umap.py:359-387) in float64: every
  gather reads the epoch-start Y, attractive pairs move both ends, each
  negative pair moves only its head, per-pair clip to [-4, 4], times alpha.
* ``optimize`` runs the epoch loop of umap.py:423-447 with the negative tails
  supplied by the caller (``neg_fn(epoch, n_neg) -> int array``), so the
  reference's draws can be injected.
"""

from __future__ import annotations

import numpy as np


def epochs_per_sample(vals: np.ndarray, n_epochs: int) -> np.ndarray:
    w = np.asarray(vals, dtype=np.float32)
    max_weight = float(w.max())
    n_samples = n_epochs * (w / max_weight)
    return np.where(n_samples > 0, n_epochs / n_samples, -1.0).astype(np.float32)


def active_sets(vals: np.ndarray, n_epochs: int):
    eps = epochs_per_sample(vals, n_epochs)
    nxt = eps.copy()
    out = []
    for epoch in range(n_epochs):
        act = np.where(nxt <= epoch)[0]
        if len(act):
            nxt[act] += eps[act]
        out.append(act.astype(np.int64))
    return out


def sgd_epoch(Y: np.ndarray, ef: np.ndarray, et: np.ndarray, neg_from: np.ndarray,
              neg_to: np.ndarray, alpha: float, a: float, b: float, dtype=np.float64) -> np.ndarray:
    Y = np.asarray(Y).astype(dtype)
    a = dtype(a)
    b = dtype(b)
    alpha = dtype(alpha)
    diff = Y[ef] - Y[et]
    d2 = np.maximum(np.sum(diff * diff, axis=1, keepdims=True), dtype(1e-6))
    coeff = -2.0 * a * b * np.power(d2, b - 1.0) / (1.0 + a * np.power(d2, b))
    pos = np.clip(coeff * diff, -4.0, 4.0) * alpha
    nd = Y[neg_from] - Y[neg_to]
    nd2 = np.maximum(np.sum(nd * nd, axis=1, keepdims=True), dtype(1e-6))
    ncoeff = 2.0 * b / ((0.001 + nd2) * (1.0 + a * np.power(nd2, b)))
    neg = np.clip(ncoeff * nd, -4.0, 4.0) * alpha
    out = Y.copy()
    np.add.at(out, ef, pos)
    np.add.at(out, et, -pos)
    np.add.at(out, neg_from, neg)
    return out


def optimize(rows, cols, vals, Y0, a: float, b: float, n_epochs: int, neg_fn,
             learning_rate: float = 1.0, negative_sample_rate: int = 5,
             epoch_range=None, callback=None, dtype=np.float64):
    rows = np.asarray(rows, dtype=np.int64)
    cols = np.asarray(cols, dtype=np.int64)
    sets = active_sets(vals, n_epochs)
    Y = np.asarray(Y0).astype(dtype)
    epochs = range(n_epochs) if epoch_range is None else epoch_range
    for epoch in epochs:
        act = sets[epoch]
        if len(act) == 0:
            continue
        ef, et = rows[act], cols[act]
        alpha = learning_rate * (1.0 - epoch / n_epochs)
        n_neg = negative_sample_rate * len(act)
        neg_from = ef[np.arange(n_neg) % len(act)]
        neg_to = np.asarray(neg_fn(epoch, n_neg), dtype=np.int64)
        Y = sgd_epoch(Y, ef, et, neg_from, neg_to, alpha, a, b, dtype=dtype)
        if callback is not None:
            callback(epoch + 1, Y)
    return Y
