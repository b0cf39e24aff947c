"""Low-dimensional membership curve 1 / (1 + a d^(2b)) fitted to the target
exp(-(d - min_dist)/spread) (1 below min_dist) — mirrors UMAP._find_ab_params,
mlx_vis/_umap/umap.py:272-296.

Gauss-Newton in float64 on 300 points of [0, 3 spread], starting at a = b = 1,
each step the least-squares solution of J step = -residual (numpy.linalg.lstsq),
at most 100 steps, stopping once |step|^2 < 1e-12.  Like the reference, a fit
that diverges surfaces numpy.linalg.LinAlgError from lstsq.  Host-side scalar
work: it runs once per fit and costs microseconds.
"""

from __future__ import annotations

import numpy as np


def find_ab_params(spread: float, min_dist: float) -> tuple[float, float]:
    x = np.linspace(0.0, 3.0 * spread, 300)
    target = np.where(x < min_dist, 1.0, np.exp(-(x - min_dist) / spread))
    log_x = np.log(np.maximum(x, 1e-20))
    a, b = 1.0, 1.0
    for _ in range(100):
        x2b = np.power(x, 2.0 * b)
        den = 1.0 + a * x2b
        resid = 1.0 / den - target
        den2 = den * den
        jac = np.column_stack([-x2b / den2, -a * 2.0 * log_x * x2b / den2])
        step = np.linalg.lstsq(jac, -resid, rcond=None)[0]
        a += step[0]
        b += step[1]
        if np.sum(step ** 2) < 1e-12:
            break
    return float(a), float(b)
