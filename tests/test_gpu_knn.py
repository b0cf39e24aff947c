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
    with pytest.raises(_lib.UmapB200Error, match="k must be <= 4096"):
        _lib.knn_brute(torch.zeros((5000, 4), device="cuda"), 4097)


@pytest.mark.parametrize("n,d,k,extra", [(3000, 64, 113, 16), (2500, 784, 300, 0), (1200, 37, 1199, 16),
                                         (41000, 16, 130, 16)])
def test_brute_long_lists_are_exact(n, d, k, extra):
    """k + extra > 128 (_knn.py has no limit on k): exact FP32-level distance tiles
    and a per-row radix select.  Against float64 exact kNN: the k-th distance per row
    within 1e-5 relative, every returned distance equal to the float64 distance of
    the returned index (1e-5 relative), indices distinct and never the row itself;
    41,000 rows take the select that re-reads the tile from memory."""
    from mlx_vis_b200 import _lib

    rng = np.random.default_rng(n + k)
    X = rng.normal(size=(n, d)).astype(np.float32)
    X[: n // 10] = X[n // 10: 2 * (n // 10)]  # exact duplicates: zero distances and ties
    Xd = torch.from_numpy(X).cuda()
    idx, dist = _lib.knn_brute(Xd, k, extra=extra)
    idx, dist = idx.cpu().numpy(), dist.cpu().numpy().astype(np.float64)
    rows = np.arange(n) if n <= 3000 else rng.choice(n, 400, replace=False)
    X64 = X.astype(np.float64)
    sq = (X64 ** 2).sum(1)
    for i in rows:
        d2 = np.maximum(sq[i] + sq - 2.0 * X64 @ X64[i], 0.0)
        d2[i] = np.inf
        kth = np.sqrt(np.partition(d2, k - 1)[k - 1])
        got = idx[i]
        assert len(set(got.tolist())) == k and i not in got
        assert np.all(np.diff(dist[i]) >= 0)
        np.testing.assert_allclose(dist[i], np.sqrt(d2[got]), rtol=1e-5, atol=1e-5 * np.sqrt(sq[i] + 1.0))
        assert abs(dist[i, -1] - kth) <= 1e-5 * (kth + np.sqrt(sq[i]) + 1e-6)
    # squared output is the square of the Euclidean one
    _, d2 = _lib.knn_brute(Xd, k, extra=extra, squared=True)
    np.testing.assert_allclose(np.sqrt(d2.cpu().numpy().astype(np.float64)), dist, rtol=1e-6, atol=1e-6)


def test_compute_knn_nndescent_branch(golden):
    """compute_knn(method="nndescent") (_knn.py:35-45): seed 42 when random_state is
    None, the NNDescent graph unchanged, squared distances for return_euclidean=False;
    the graph agrees with the reference's NNDescent on the same data and seed."""
    from mlx_vis_b200 import NNDescent, datasets
    from mlx_vis_b200._knn import compute_knn

    Xn = datasets.gaussian_mixture(3000, 32, seed=2)
    idx, dist = compute_knn(Xn, 15, method="nndescent")
    assert idx.dtype == np.int32 and dist.dtype == np.float32 and idx.shape == (3000, 15)
    ref_i, ref_d = NNDescent(k=15, random_state=42).build(Xn)
    assert np.array_equal(idx, ref_i) and np.array_equal(dist, ref_d)
    idx_sq, d2 = compute_knn(Xn, 15, method="nndescent", return_euclidean=False)
    assert np.array_equal(idx_sq, idx) and np.array_equal(d2, dist ** 2)
    idx7, _ = compute_knn(Xn, 15, method="nndescent", random_state=7)
    assert not np.array_equal(idx7, idx)  # the seed reaches NNDescent
    g = golden("nnd_gauss")
    assert np.mean(idx == g["idx_it20"]) > 0.99


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


def exact_knn_f64_cuda(X: np.ndarray, k: int, cand: int = 48, chunk: int = 2048):
    """Exact kNN of every row in float64 on the GPU (test-side checker, torch
    float64): expanded-form distances pick the best `cand` candidates, whose
    distances are then recomputed as sum (x_i - x_j)^2; (distance, index) order."""
    Xd = torch.from_numpy(X).cuda().double()
    n = Xd.shape[0]
    sq = (Xd * Xd).sum(1)
    out_i = torch.empty((n, k), dtype=torch.int64, device="cuda")
    out_d = torch.empty((n, k), dtype=torch.float64, device="cuda")
    for s in range(0, n, chunk):
        e = min(s + chunk, n)
        D = sq[s:e, None] + sq[None, :] - 2.0 * (Xd[s:e] @ Xd.T)
        D[torch.arange(e - s, device="cuda"), torch.arange(s, e, device="cuda")] = float("inf")
        c = torch.topk(D, cand, dim=1, largest=False).indices
        d2 = ((Xd[c] - Xd[s:e, None, :]) ** 2).sum(-1)
        # order by (distance, index): index breaks exact ties
        key = torch.argsort(c, dim=1, stable=True)
        c, d2 = torch.gather(c, 1, key), torch.gather(d2, 1, key)
        o = torch.argsort(d2, dim=1, stable=True)[:, :k]
        out_i[s:e] = torch.gather(c, 1, o)
        out_d[s:e] = torch.gather(d2, 1, o)
    return out_i.cpu().numpy(), out_d.cpu().numpy()


def test_brute_tile_paths_agree_at_scale(tile_path):
    """The 20000 x 784 exact-kNN workload (several row blocks per unit, candidate
    slots > 1): EVERY row against the float64 exact kNN, ties within 1e-6 relative
    distance allowed to swap."""
    from mlx_vis_b200 import datasets

    X = datasets.prototype_mixture(20000, 784, seed=0)
    idx, dist = run_knn(X, 15)
    want_i, want_d2 = exact_knn_f64_cuda(X, 15)
    Xt = torch.from_numpy(X).cuda().double()
    ours_d2 = ((Xt[torch.from_numpy(idx).cuda().long()] - Xt[:, None, :]) ** 2).sum(-1).cpu().numpy()
    assert np.all(idx != np.arange(len(X))[:, None])
    assert all(len(set(r)) == 15 for r in idx)
    # the sorted distance profile equals the exact one up to ties
    assert np.all(np.abs(ours_d2 - want_d2) <= TIE * np.maximum(want_d2, 1e-12) + 1e-12)
    np.testing.assert_allclose(dist, np.sqrt(want_d2), rtol=2e-6, atol=1e-6)
    # indices equal the exact ones wherever the distance is not tied
    agree = np.mean(idx == want_i)
    assert agree > 0.999, agree


@pytest.mark.parametrize("n,d,parts", [(3000, 64, 3), (20000, 784, 2), (1000, 130, 7)])
def test_brute_rows_blocks_reassemble_the_full_result(n, d, parts, tile_path):
    """umapb_knn_brute_rows on the blocks of a row split (the per-rank work of the
    sharded kNN) gives the rows of umapb_knn_brute: same indices, same distances."""
    from mlx_vis_b200 import _lib
    from mlx_vis_b200._distributed import knn_brute_sharded, row_blocks

    X = np.random.default_rng(n + d).normal(size=(n, d)).astype(np.float32)
    Xd = torch.from_numpy(X).cuda()
    ref_i, ref_d = _lib.knn_brute(Xd, 15)
    got = [_lib.knn_brute_rows(Xd, 15, b, c) for b, c in row_blocks(n, parts)]
    idx = torch.cat([g[0] for g in got])
    dst = torch.cat([g[1] for g in got])
    assert torch.equal(idx, ref_i)
    torch.testing.assert_close(dst, ref_d, rtol=1e-6, atol=1e-6)
    # one process, no group: the sharded entry runs the whole range
    i1, d1 = knn_brute_sharded(Xd, 15)
    assert torch.equal(i1, ref_i)


def test_brute_rows_argument_errors():
    from mlx_vis_b200 import _lib

    X = torch.zeros((100, 4), device="cuda")
    with pytest.raises(_lib.UmapB200Error, match="query rows"):
        _lib.knn_brute_rows(X, 5, 90, 20)
    with pytest.raises(_lib.UmapB200Error, match="query rows"):
        _lib.knn_brute_rows(X, 5, -1, 2)
