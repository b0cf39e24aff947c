"""Whole-fit CPU baseline (test infrastructure, and the CPU leg of bench.py).

The reference's own MLX CPU backend cannot be installed offline, so the
baseline is this oracle (a NumPy restatement of the reference's algorithm) run
on the host cores.  A 70,000 x 784 fit does not fit the CPU budget of a
benchmark run (its NNDescent gathers alone are ~56 GB per iteration), so each
stage is timed on a bounded sample of the same workload and extrapolated:

  kNN (NNDescent, nndescent.py:34-403)  cost per row-iteration x n x iterations
  fuzzy set (umap.py:199-270)            linear in n
  spectral init (umap.py:298-357)        linear in the edge count
  layout (umap.py:389-449)               linear in positive-edge updates

Returned figures name the sample and the scale factors.
"""

from __future__ import annotations

import os
import time

import numpy as np

from oracle import fuzzy as ofz
from oracle import layout as olay
from oracle import nndescent as onnd
from oracle import spectral as ospec


def edge_updates(vals: np.ndarray, n_epochs: int) -> int:
    """Positive-edge updates of a whole optimize_layout run (umap.py:401-414)."""
    return int(sum(len(a) for a in olay.active_sets(vals, n_epochs)))


def estimate_fit(n_full: int, make_sample, sample_n: int, n_epochs: int = 500, k: int = 15, a: float = 1.5769,
                 b: float = 0.8951, seed: int = 0) -> dict:
    """Times each stage of a fit on ``make_sample(sample_n)`` and scales it to n_full."""
    Xs = make_sample(sample_n)
    out = {"sample": f"{sample_n} x {Xs.shape[1]} rows of the same generator, all stages, {n_epochs} epochs",
           "threads": os.cpu_count()}
    t = time.perf_counter()
    (idx, dist), log = onnd.build(Xs, k=k, random_state=42, history=True)
    t_knn = time.perf_counter() - t
    t = time.perf_counter()
    (rows, cols, vals), _ = ofz.fuzzy_simplicial_set(idx, dist, n_epochs, dtype=np.float32)
    t_fuzzy = time.perf_counter() - t
    rng = np.random.default_rng(seed)
    V0 = rng.standard_normal((sample_n, 3)).astype(np.float32)
    t = time.perf_counter()
    Y0 = ospec.spectral_init(rows, cols, vals, sample_n, V0, seed, dtype=np.float32)
    t_spec = time.perf_counter() - t
    t = time.perf_counter()
    olay.optimize(rows, cols, vals, Y0, a, b, n_epochs,
                  lambda e, nn: rng.integers(0, sample_n, nn), dtype=np.float32)
    t_layout = time.perf_counter() - t
    upd_sample = edge_updates(vals, n_epochs)
    scale_rows = n_full / sample_n
    upd_full = upd_sample * scale_rows  # the same degree distribution per row
    est = {"knn": t_knn * scale_rows, "fuzzy": t_fuzzy * scale_rows, "init": t_spec * scale_rows,
           "layout": t_layout * (upd_full / max(upd_sample, 1))}
    out.update(stage_s_sample={"knn": t_knn, "fuzzy": t_fuzzy, "init": t_spec, "layout": t_layout},
               stage_s_full=est, fit_s_full=sum(est.values()), edge_updates_full=upd_full,
               edge_updates_sample=upd_sample, nnd_iterations_sample=len(log), cpu_s=t_knn + t_fuzzy + t_spec + t_layout)
    return out
