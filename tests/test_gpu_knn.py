"""Brute-force kNN on the GPU (tcgen05 BF16 tiles + fused top-(k+16) + exact FP32
rerank) against the float64 oracle and the reference's own output.

Parity bar: the index sets equal the float64 exact kNN except where two
candidates' exact distances differ by less than 1e-6 relative (ties); distances
within 1e-6 relative of float64.  Disagreements with the reference's float32
expanded-form path must be explained by that path's own rounding error.
"""

import numpy as np
import pytest
import torch

from oracle import knn as oknn

pytestmark = pytest.mark.gpu
TIE = 2e-6  # on squared distances: 1e-6 relative on the Euclidean distance


def run_knn(X, k, extra=16, squared=False):
    from mlx_vis_b200 import _lib

    idx, dist = _lib.knn_brute(torch.from_numpy(np.ascontiguousarray(X, dtype=np.float32)).cuda(), k, extra=extra,
                               squared=squared)
    return idx.cpu().numpy(), dist.cpu().numpy()


def assert_exact_knn(X, idx, dist, k, squared=False):
    """Tie-aware comparison with the float64 oracle."""
    n = X.shape[0]
    ref_idx, ref_d2 = oknn.knn_exact_f64(X, k)
    assert idx.shape == (n, k) and dist.shape == (n, k)
    assert np.all((idx >= 0) & (idx < n))
    assert np.all(idx != np.arange(n)[:, None]), "self must be excluded"
    for r in range(n):
        assert len(set(idx[r])) == k, f"duplicate neighbours in row {r}"
    # exact distances of our neighbours
    ours_d2 = oknn.sqdist_f64(X, np.arange(n), idx)
    assert np.all(np.diff(ours_d2, axis=1) >= -TIE * np.maximum(ours_d2[:, 1:], 1e-30)), "not ascending"
    # sorted distance profile must equal the exact one (ties allowed to swap ids)
    scale = np.maximum(ref_d2, 1e-12)
    assert np.all(np.abs(ours_d2 - ref_d2) <= TIE * scale + 1e-12), "distance profile differs from exact kNN"
    mism = idx != ref_idx
    if mism.any():  # every id mismatch must sit inside a tie group
        rr, cc = np.nonzero(mism)
        kth = ref_d2[rr, cc]
        assert np.all(np.abs(ours_d2[rr, cc] - kth) <= TIE * np.maximum(kth, 1e-12) + 1e-12)
    want = ref_d2 if squared else np.sqrt(ref_d2)
    np.testing.assert_allclose(dist, want, rtol=2e-6, atol=1e-6)


@pytest.mark.parametrize("name,fixture", [("knn_brute_gauss", "gauss2000"), ("knn_brute_proto", "proto1500")])
def test_brute_matches_exact_and_reference(name, fixture, golden, request):
    X = request.getfixturevalue(fixture)
    g = golden(name)
    idx, dist = run_knn(X, 15)
    assert_exact_knn(X, idx, dist, 15)
    # against the reference's own float32 expanded-form result
    agree = np.mean([len(set(a) & set(b)) / 15 for a, b in zip(idx, g["idx"])])
    assert agree > 0.999
    rows = np.nonzero([set(a) != set(b) for a, b in zip(idx, g["idx"])])[0]
    for r in rows:  # each reference disagreement must be within its own float32 error
        theirs = sorted(set(g["idx"][r]) - set(idx[r]))
        mine = sorted(set(idx[r]) - set(g["idx"][r]))
        dt = oknn.sqdist_f64(X, np.array([r]), np.array([theirs]))[0]
        dm = oknn.sqdist_f64(X, np.array([r]), np.array([mine]))[0]
        sq = float(np.sum(X[r].astype(np.float64) ** 2))
        bound = 64 * np.finfo(np.float32).eps * (2 * sq + 1.0)
        assert np.max(np.abs(dt - dm)) <= bound
    np.testing.assert_allclose(dist, g["dist"], rtol=1e-4, atol=1e-4)


@pytest.mark.parametrize("n,d,k", [(2, 3, 1), (3, 1, 2), (17, 5, 16), (129, 65, 15), (257, 130, 15),
                                   (300, 784, 15), (1000, 7, 15), (5000, 32, 15)])
def test_brute_ragged_shapes(n, d, k):
    rng = np.random.default_rng(n * 1000 + d)
    X = rng.normal(size=(n, d)).astype(np.float32)
    idx, dist = run_knn(X, k)
    assert_exact_knn(X, idx, dist, k)


@pytest.mark.parametrize("k,extra", [(40, 16), (100, 16), (1, 16), (8, 60)])
def test_brute_candidate_list_sizes(k, extra):
    X = np.random.default_rng(k).normal(size=(700, 24)).astype(np.float32)
    idx, dist = run_knn(X, k, extra=extra)
    assert_exact_knn(X, idx, dist, k)


def test_brute_squared_and_duplicates():
    rng = np.random.default_rng(5)
    X = rng.normal(size=(400, 16)).astype(np.float32)
    X[200:260] = X[0:60]  # exact duplicates: zero distances and equal-distance groups
    idx, d2 = run_knn(X, 15, squared=True)
    assert_exact_knn(X, idx, d2, 15, squared=True)
    assert np.all(d2[:60, 0] == 0.0) and np.all(idx[:60, 0] == np.arange(200, 260))


def test_brute_argument_errors():
    from mlx_vis_b200 import _lib

    X = torch.zeros((10, 4), device="cuda")
    with pytest.raises(_lib.UmapB200Error, match="k <= n-1"):
        _lib.knn_brute(X, 10)
    with pytest.raises(_lib.UmapB200Error, match="k <= n-1"):
        _lib.knn_brute(X, 0)
    with pytest.raises(_lib.UmapB200Error, match="<= 128"):
        _lib.knn_brute(torch.zeros((500, 4), device="cuda"), 120, extra=16)


def test_compute_knn_plug_point(gauss2000, golden):
    from mlx_vis_b200._knn import compute_knn

    idx, dist = compute_knn(gauss2000, 15, method="brute")
    assert idx.dtype == np.int32 and dist.dtype == np.float32
    idx2, d2 = compute_knn(gauss2000, 15, method="brute", return_euclidean=False)
    np.testing.assert_allclose(np.sqrt(d2), dist, rtol=1e-6)
    assert np.mean(idx == golden("knn_brute_gauss")["idx"]) > 0.999


@pytest.fixture(params=["pair", "single"])
def tile_path(request, monkeypatch):
    """L <= 32 runs on CTA pairs (256-row tiles, tcgen05 cta_group::2) unless
    UMAPB_KNN_PAIR=0 selects the one-CTA 128-row tiles; both must be exact."""
    monkeypatch.setenv("UMAPB_KNN_PAIR", "1" if request.param == "pair" else "0")
    return request.param


@pytest.mark.parametrize("n,d,k", [(2, 3, 1), (129, 65, 15), (255, 40, 15), (256, 64, 15), (257, 130, 15),
                                   (300, 784, 15), (383, 17, 16), (513, 100, 15), (5000, 32, 15)])
def test_brute_tile_paths_ragged(n, d, k, tile_path):
    rng = np.random.default_rng(n * 7 + d)
    X = rng.normal(size=(n, d)).astype(np.float32)
    idx, dist = run_knn(X, k)
    assert_exact_knn(X, idx, dist, k)


def test_brute_tile_paths_agree_at_scale(tile_path):
    """20000 x 784 (several row blocks per unit, candidate slots > 1): sampled
    rows against the float64 exact kNN."""
    from mlx_vis_b200 import datasets

    X = datasets.prototype_mixture(20000, 784, seed=0)
    idx, dist = run_knn(X, 15)
    rows = np.random.default_rng(1).choice(X.shape[0], 300, replace=False)
    Xd = X.astype(np.float64)
    sq = np.sum(Xd * Xd, axis=1)
    D = sq[rows, None] + sq[None, :] - 2.0 * (Xd[rows] @ Xd.T)
    D[np.arange(len(rows)), rows] = np.inf
    cand = np.argpartition(D, 40, axis=1)[:, :40]  # exact top-15 lies among them
    for i, r in enumerate(rows):
        c = cand[i]
        d2 = np.sum((Xd[c] - Xd[r]) ** 2, axis=1)
        o = np.lexsort((c, d2))[:15]
        want = d2[o]
        ours = np.sum((Xd[idx[r]] - Xd[r]) ** 2, axis=1)
        assert np.all(np.abs(ours - want) <= TIE * np.maximum(want, 1e-12) + 1e-12), r
        np.testing.assert_allclose(dist[r], np.sqrt(want), rtol=2e-6, atol=1e-6)
