"""Input normalisation before the kNN step — mirrors mlx_vis/_normalize.py:6-33.

``False``/``None`` pass the data through, ``True``/``"standard"`` z-score each
feature (population std + 1e-8), ``"minmax"`` scales each feature to [0, 1]
(range + 1e-8); anything else raises ``ValueError`` like the reference.
Host NumPy float32, as in the reference.
"""

from __future__ import annotations

import numpy as np


def normalize_input(X: np.ndarray, method) -> np.ndarray:
    if method is None or method is False:
        return X
    if isinstance(method, str) and method == "":
        return X
    if method is True or method == "standard":
        mu = X.mean(axis=0)
        sd = X.std(axis=0) + 1e-8
        return (X - mu) / sd
    if method == "minmax":
        lo = X.min(axis=0)
        span = X.max(axis=0) - lo + 1e-8
        return (X - lo) / span
    raise ValueError(f"Unknown normalize method: {method}")
