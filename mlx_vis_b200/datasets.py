"""Seeded synthetic inputs for the UMAP workloads.

Fashion-MNIST (the reference README's 70,000 x 784 benchmark, README.md:161-166)
is not available offline, so every workload runs on seeded synthetic mixtures
with the same shapes:

* ``gaussian_mixture``   - 2000 x 64, 10 isotropic Gaussians (centres ~ N(0, 16 I),
  sigma 1, equal weights): the small CPU-runnable workload.
* ``prototype_mixture``  - pixel-like rows: one of 10 prototypes in [0, 1]^d with
  about half the entries zero, plus N(0, 0.1^2) noise, clipped to [0, 1]
  (20000 x 784 exact-kNN workload, 70000 x 784 full pipeline).
* ``anisotropic_mixture`` - 1,000,000 x 128, 100 rotated anisotropic Gaussians with
  per-axis sigma ~ U(0.3, 2) and Dirichlet(2) cluster sizes.

All generators use ``numpy.random.default_rng`` so a (seed, shape) pair always
produces the same float32 array on every machine.
"""

from __future__ import annotations

import numpy as np


def _equal_labels(n: int, n_classes: int, rng: np.random.Generator) -> np.ndarray:
    labels = np.arange(n, dtype=np.int32) % n_classes
    rng.shuffle(labels)
    return labels


def gaussian_mixture(n: int = 2000, d: int = 64, n_centers: int = 10,
                     center_std: float = 4.0, sigma: float = 1.0, seed: int = 0,
                     return_labels: bool = False):
    """Equal-weight isotropic Gaussian mixture, float32 (n, d)."""
    rng = np.random.default_rng(seed)
    centers = rng.standard_normal((n_centers, d)) * center_std
    labels = _equal_labels(n, n_centers, rng)
    X = centers[labels] + rng.standard_normal((n, d)) * sigma
    X = X.astype(np.float32)
    return (X, labels) if return_labels else X


def make_prototypes(d: int = 784, n_classes: int = 10, proto_seed: int = 0) -> np.ndarray:
    """Prototype vectors in [0, 1]^d with roughly 50% of the entries set to 0."""
    rng = np.random.default_rng(10_000 + proto_seed)
    protos = rng.random((n_classes, d))
    protos[rng.random((n_classes, d)) < 0.5] = 0.0
    return protos.astype(np.float32)


def prototype_mixture(n: int = 20000, d: int = 784, n_classes: int = 10,
                      noise: float = 0.1, seed: int = 0, proto_seed: int | None = None,
                      return_labels: bool = False):
    """Pixel-like prototype mixture, float32 (n, d) with values in [0, 1].

    ``proto_seed`` selects the prototypes (defaults to ``seed``) and ``seed`` the
    samples, so a family of datasets can share prototypes while drawing fresh rows.
    """
    protos = make_prototypes(d, n_classes, seed if proto_seed is None else proto_seed)
    rng = np.random.default_rng(seed)
    labels = _equal_labels(n, n_classes, rng)
    X = protos[labels]
    X = X + (rng.standard_normal((n, d), dtype=np.float32) * np.float32(noise))
    np.clip(X, 0.0, 1.0, out=X)
    X = X.astype(np.float32, copy=False)
    return (X, labels) if return_labels else X


def anisotropic_mixture(n: int = 1_000_000, d: int = 128, n_clusters: int = 100,
                        center_std: float = 8.0, seed: int = 0, param_seed: int | None = None,
                        return_labels: bool = False):
    """Rotated anisotropic Gaussian mixture: cluster sizes ~ Dirichlet(2), centres
    ~ N(0, center_std^2 I), random orthogonal rotations, per-axis sigma ~ U(0.3, 2).

    ``param_seed`` fixes the clusters (sizes, centres, rotations, scales; defaults to
    ``seed``) and ``seed`` the sampled rows, so several draws can share one
    distribution."""
    prng = np.random.default_rng(seed if param_seed is None else param_seed)
    sizes = prng.dirichlet(np.full(n_clusters, 2.0))
    centers = (prng.standard_normal((n_clusters, d)) * center_std).astype(np.float32)
    rots = [np.linalg.qr(prng.standard_normal((d, d)))[0].astype(np.float32) for _ in range(n_clusters)]
    scales = prng.uniform(0.3, 2.0, (n_clusters, d)).astype(np.float32)
    rng = np.random.default_rng((seed, 1))
    counts = np.floor(sizes * n).astype(np.int64)
    counts[: n - counts.sum()] += 1
    labels = np.repeat(np.arange(n_clusters, dtype=np.int32), counts)
    rng.shuffle(labels)
    X = np.empty((n, d), dtype=np.float32)
    for c in range(n_clusters):
        rows = np.nonzero(labels == c)[0]
        z = rng.standard_normal((rows.size, d), dtype=np.float32) * scales[c]
        X[rows] = z @ rots[c].T + centers[c]
    return (X, labels) if return_labels else X
