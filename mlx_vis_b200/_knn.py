"""Shared kNN entry point — mirrors ``compute_knn`` of mlx_vis/_knn.py:7-88.

``method="auto"`` picks brute force for n <= 20000 and NNDescent above
(_knn.py:32-33); ``"nndescent"`` runs NNDescent with random_state 42 when none
is given (_knn.py:37-41); any other string falls through to brute force, as in
the reference (_knn.py:35, 47).  Brute force is the tcgen05 kernel of
libumap_b200 (BF16 distance tiles, fused top-(k+16), exact FP32 rerank).
"""

from __future__ import annotations

import numpy as np
import torch

from mlx_vis_b200 import _lib
from mlx_vis_b200._device import to_device_f32, to_host

AUTO_BRUTE_MAX_N = 20000
RERANK_EXTRA = 16


def resolve_method(method: str, n: int) -> str:
    if method == "auto":
        return "brute" if n <= AUTO_BRUTE_MAX_N else "nndescent"
    return "nndescent" if method == "nndescent" else "brute"


def knn_device(X: torch.Tensor, k: int, method: str = "auto", verbose: bool = False, random_state=None,
               squared: bool = False):
    """kNN on device: (idx int32 (n,k), dist float32 (n,k)) CUDA tensors; Euclidean
    distances unless ``squared`` (brute force only; NNDescent returns Euclidean)."""
    n = X.shape[0]
    m = resolve_method(method, n)
    if m == "nndescent":
        from mlx_vis_b200._nndescent.nndescent import NNDescent

        nn = NNDescent(k=k, verbose=verbose, random_state=random_state if random_state is not None else 42)
        return nn.build_device(X)
    return _lib.knn_brute(X, k, extra=RERANK_EXTRA, squared=squared)


def compute_knn(X, k, method="auto", verbose=False, random_state=None, return_euclidean=True):
    """Same signature and outputs as the reference: host (indices int32, distances float32)."""
    Xd = to_device_f32(X)
    brute = resolve_method(method, Xd.shape[0]) == "brute"
    idx, dist = knn_device(Xd, int(k), method=method, verbose=verbose, random_state=random_state,
                           squared=brute and not return_euclidean)
    dist_np = to_host(dist).astype(np.float32)
    if not return_euclidean and not brute:
        dist_np = dist_np ** 2  # the reference squares NNDescent's Euclidean output (_knn.py:43-44)
    return to_host(idx).astype(np.int32), dist_np
