"""Embedding quality metrics on the GPU (evaluation utilities, not the UMAP path).

``trustworthiness`` follows sklearn.manifold.trustworthiness exactly (Euclidean
input distances with the diagonal excluded, 1-based ranks, the embedding's
k nearest neighbours without self, penalty max(0, rank - k), normalisation
2 / (n k (2n - 3k - 1))), computed in row chunks with float64 input distances so
ranks are exact; usable at sizes where the sklearn version runs out of memory.
"""

from __future__ import annotations

import numpy as np
import torch


def trustworthiness(X, Y, n_neighbors: int = 15, chunk: int = 1024) -> float:
    dev = torch.device("cuda")
    Xt = torch.as_tensor(np.asarray(X), dtype=torch.float64, device=dev)
    Yt = torch.as_tensor(np.asarray(Y), dtype=torch.float32, device=dev)
    n, k = Xt.shape[0], n_neighbors
    if not 1 <= k < n / 2:
        raise ValueError("n_neighbors must be in [1, n/2)")
    sqx = (Xt * Xt).sum(1)
    sqy = (Yt * Yt).sum(1)
    total = 0.0
    ar = torch.arange(n, device=dev)
    for s in range(0, n, chunk):
        e = min(s + chunk, n)
        rows = ar[s:e]
        dx = sqx[s:e, None] + sqx[None, :] - 2.0 * (Xt[s:e] @ Xt.T)
        dx[torch.arange(e - s, device=dev), rows] = float("inf")
        order = torch.argsort(dx, dim=1, stable=True)
        ranks = torch.empty_like(order)
        ranks.scatter_(1, order, ar.expand(e - s, n) + 1)
        dy = sqy[s:e, None] + sqy[None, :] - 2.0 * (Yt[s:e] @ Yt.T)
        dy[torch.arange(e - s, device=dev), rows] = float("inf")
        nn = torch.topk(dy, k, dim=1, largest=False).indices
        r = torch.gather(ranks, 1, nn) - k
        total += float(r.clamp_min(0).sum().item())
    return 1.0 - total * (2.0 / (n * k * (2.0 * n - 3.0 * k - 1.0)))
