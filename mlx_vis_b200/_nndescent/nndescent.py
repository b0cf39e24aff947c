"""NNDescent on one B200 — drop-in for ``mlx_vis.NNDescent`` (mlx_vis/_nndescent/nndescent.py:14-403)."""

from __future__ import annotations

import numpy as np
import torch

from mlx_vis_b200._device import to_device_f32, to_host


class NNDescent:
    """Approximate k-NN graph via NNDescent (constructor mirrors nndescent.py:17-32)."""

    def __init__(self, k: int = 15, n_iters: int = 20, max_candidates: int | None = None, delta: float = 0.015,
                 random_state: int | None = None, verbose: bool = False):
        self.k = k
        self.n_iters = n_iters
        self.max_candidates = max_candidates
        self.delta = delta
        self.random_state = random_state
        self.verbose = verbose
        self.neighbor_graph = None

    def build(self, X) -> tuple[np.ndarray, np.ndarray]:
        idx, dist = self.build_device(to_device_f32(X))
        self.neighbor_graph = (to_host(idx).astype(np.int32), to_host(dist).astype(np.float32))
        return self.neighbor_graph

    def build_device(self, X: torch.Tensor):
        raise NotImplementedError("NNDescent kernels are not built yet")
