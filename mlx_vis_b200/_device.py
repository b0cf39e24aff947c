"""Device selection and input conversion shared by the estimators."""

from __future__ import annotations

import numpy as np
import torch


def device() -> torch.device:
    if not torch.cuda.is_available():
        raise RuntimeError("mlx_vis_b200 needs a CUDA device (B200, sm_100a); none is visible")
    return torch.device("cuda", torch.cuda.current_device())


def to_device_f32(X, dev: torch.device | None = None) -> torch.Tensor:
    """numpy / array-like / torch input -> contiguous float32 (n, d) CUDA tensor.

    Host arrays go through pinned memory so the upload is one DMA."""
    dev = dev or device()
    if isinstance(X, torch.Tensor):
        t = X.detach()
        if t.dtype != torch.float32:
            t = t.float()
        return t.to(dev, non_blocking=True).contiguous()
    a = np.ascontiguousarray(np.asarray(X, dtype=np.float32))
    if a.ndim != 2:
        raise ValueError(f"expected a 2-D array (n_samples, n_features), got shape {a.shape}")
    host = torch.from_numpy(a)
    if a.nbytes >= (1 << 20):
        host = host.pin_memory()
    return host.to(dev, non_blocking=True)


def to_host(t: torch.Tensor) -> np.ndarray:
    return t.detach().cpu().numpy()
