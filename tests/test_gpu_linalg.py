"""Split-precision tensor-core products (umapb_split3 + umapb_gemm_split3), column
means, the key sort, and the PCA preprocessing built on them (umap.py:92-113),
against float64 NumPy and the reference's own PCA output."""

import numpy as np
import pytest
import torch

from oracle import pca as opca

pytestmark = pytest.mark.gpu


def cuda(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("M,K,N", [(1, 1, 1), (70, 33, 5), (128, 64, 128), (300, 784, 100), (1000, 130, 300),
                                   (4097, 784, 129)])
def test_split3_matmul_has_fp32_level_error(M, K, N):
    """A @ B from three BF16 parts per value and six tcgen05 products: the error
    against float64 stays at the level of an FP32 GEMM (a few 2^-24 of sum |a||b|)."""
    from mlx_vis_b200 import _lib

    rng = np.random.default_rng(M + K + N)
    A = rng.normal(size=(M, K)).astype(np.float32)
    B = rng.normal(size=(K, N)).astype(np.float32)
    C = _lib.matmul(cuda(A), cuda(B)).cpu().numpy()
    ref = A.astype(np.float64) @ B.astype(np.float64)
    scale = np.abs(A).astype(np.float64) @ np.abs(B).astype(np.float64)
    err = np.abs(C - ref) / np.maximum(scale, 1e-30)
    assert err.max() < 5e-6, err.max()
    # a plain FP32 product of the same data for scale: its error is of the same order
    f32 = np.abs(A @ B - ref) / np.maximum(scale, 1e-30)
    assert err.max() < 20 * max(f32.max(), 6e-8)


def test_split3_transpose_and_mean_with_k_slices():
    """Covariance form (X - mu)^T (X - mu) with the K range cut into slices."""
    from mlx_vis_b200 import _lib

    rng = np.random.default_rng(5)
    X = (rng.normal(size=(3001, 70)) * 3 + 5).astype(np.float32)
    Xd = cuda(X)
    mu = _lib.colmean(Xd)
    np.testing.assert_allclose(mu.cpu().numpy(), X.astype(np.float64).mean(0), rtol=1e-6, atol=1e-6)
    XT3, kp = _lib.split3(Xd, mu=mu, transpose=True)
    assert XT3.shape == (70, 3 * kp) and kp % 64 == 0 and kp >= 3001
    Xc = X.astype(np.float64) - mu.cpu().numpy().astype(np.float64)
    ref = Xc.T @ Xc / 3000
    # default: slices of at most 1024 rows of K, summed in FP64
    for ks in (None, 7):
        cov = _lib.gemm_split3(XT3, XT3, kp, ksplit=ks, scale=1.0 / 3000).cpu().numpy()
        assert np.abs(cov - ref).max() < 1e-5 * np.abs(ref).max(), ks
    # one accumulator over all 3001 rows: the tensor cores' FP32 additions drift
    # with K on the all-positive diagonal, still within 1e-4
    cov = _lib.gemm_split3(XT3, XT3, kp, ksplit=1, scale=1.0 / 3000).cpu().numpy()
    assert np.abs(cov - ref).max() < 1e-4 * np.abs(ref).max()


@pytest.mark.parametrize("n", [1, 5, 1023, 1024, 1025, 70000, 5_000_003])
def test_sort_keys_is_a_stable_argsort(n):
    """Also covers the exclusive scan of the tile histograms: 256 x tiles counts, one
    block up to 16 K of them, several blocks (with several passes each) above."""
    from mlx_vis_b200 import _lib

    rng = np.random.default_rng(n)
    keys = rng.normal(size=n).astype(np.float32)
    keys[: n // 3] = np.round(keys[: n // 3], 1)  # many exact ties
    if n > 4:
        keys[:2] = [0.0, 0.0]
        keys[2:4] = [np.inf, -np.inf]
    order = _lib.sort_keys(cuda(keys)).cpu().numpy()
    want = np.argsort(keys, kind="stable")
    assert np.array_equal(order, want)
    assert sorted(order.tolist()) == list(range(n))
    same = keys[order][1:] == keys[order][:-1]
    assert np.all(order[1:][same] > order[:-1][same]) or n < 2  # ties keep their index order


def test_sort_keys_reads_a_strided_column():
    from mlx_vis_b200 import _lib

    M = np.random.default_rng(3).normal(size=(5000, 7)).astype(np.float32)
    Md = cuda(M)
    order = _lib.sort_keys(Md[:, 3]).cpu().numpy()
    assert np.array_equal(order, np.argsort(M[:, 3], kind="stable"))


def test_pca_matches_the_reference(manifest, golden):
    """UMAP(pca_dim=20) preprocessing: the reference's X_for_knn (its own code on the
    NumPy mlx shim, umap.py:92-113) and the float64 oracle, per column up to sign."""
    from mlx_vis_b200 import UMAP
    from mlx_vis_b200.datasets import prototype_mixture

    X = prototype_mixture(1000, 784, seed=4)
    u = UMAP(pca_dim=20, random_state=0)
    got = u._pca(cuda(X)).cpu().numpy().astype(np.float64)
    ref = golden("pca_proto")["X_pca"].astype(np.float64)
    o, w, _ = opca.pca(X, 20)
    scale = np.abs(o).max()
    assert np.abs(opca.align_signs(o, got) - o).max() < 1e-4 * scale
    assert np.abs(opca.align_signs(ref, got) - ref).max() < 1e-3 * scale
    np.testing.assert_allclose(u.pca_eigenvalues_[-20:], w[-20:], rtol=1e-4)


def test_pca_fit_runs_and_keeps_neighbourhoods():
    from sklearn.manifold import trustworthiness

    from mlx_vis_b200 import UMAP
    from mlx_vis_b200.datasets import prototype_mixture

    X = prototype_mixture(3000, 784, seed=6)
    Y = UMAP(pca_dim=50, n_epochs=200, knn_method="brute", random_state=0).fit_transform(X)
    Y0 = UMAP(n_epochs=200, knn_method="brute", random_state=0).fit_transform(X)
    assert Y.shape == (3000, 2) and np.isfinite(Y).all()
    t, t0 = trustworthiness(X, Y, n_neighbors=15), trustworthiness(X, Y0, n_neighbors=15)
    assert t > t0 - 0.01, (t, t0)


def test_nndescent_projections_match_numpy():
    """X @ P (100-d) and X @ P2 (300-d) of the random start through the split GEMM,
    within FP32-level error of NumPy's float64 product of the same P, P2."""
    from mlx_vis_b200 import _lib
    from mlx_vis_b200._nndescent.nndescent import random_start
    from mlx_vis_b200.datasets import prototype_mixture

    X = prototype_mixture(2000, 784, seed=3)
    _, P, P2 = random_start(2000, 15, 784, 42)
    for Pm in (P, P2):
        got = _lib.matmul(cuda(X), cuda(Pm)).cpu().numpy()
        ref = X.astype(np.float64) @ Pm.astype(np.float64)
        scale = np.abs(X).astype(np.float64) @ np.abs(Pm).astype(np.float64)
        assert (np.abs(got - ref) / scale).max() < 5e-6
