"""NNDescent on the GPU against the NumPy oracle of the reference algorithm
(same NumPy random start and projections) and the reference's golden graphs.

The GPU and the oracle make the same choices except where float rounding orders
two nearly equal distances differently (GPU dot products are summed in another
order, FP16 iterations round those sums), so graphs agree row-set-wise to
within a fraction of a percent and the per-iteration change counts track."""

import numpy as np
import pytest
import torch

from oracle import knn as oknn
from oracle import nndescent as onnd

pytestmark = pytest.mark.gpu


def recall(idx, ref_idx):
    return float(np.mean([len(set(a) & set(b)) / len(a) for a, b in zip(idx, ref_idx)]))


@pytest.mark.parametrize("name,gen", [("nnd_gauss", ("gaussian_mixture", 3000, 32, 2)),
                                      ("nnd_proto", ("prototype_mixture", 2000, 784, 3))])
def test_nndescent_tracks_oracle_and_reference(name, gen, golden):
    from mlx_vis_b200 import NNDescent, datasets

    X = getattr(datasets, gen[0])(gen[1], gen[2], seed=gen[3])
    g = golden(name)
    its = sorted(int(k[6:]) for k in g if k.startswith("idx_it"))
    for t in its:
        nn = NNDescent(k=15, random_state=42, n_iters=t)
        idx, dist = nn.build(X)
        (oi, od), olog = onnd.build(X, k=15, random_state=42, n_iters=t, history=True)
        agree = recall(idx, oi)
        assert agree > 0.99, (t, agree)
        ours = [h["changed"] for h in nn.history_]
        theirs = [l["changed"] for l in olog]
        assert len(ours) == len(theirs), (ours, theirs)
        np.testing.assert_allclose(ours, theirs, rtol=0.02, atol=20)
        gi = g[f"idx_it{t}"].astype(np.int32)
        assert recall(idx, gi) > 0.98
        # distances: the space of the iteration that produced them (the 100-d
        # projection after iteration 1, FP16-rounded dots in iterations 2-5, FP32
        # afterwards), as in the reference; compare where the lists agree
        same = idx == oi
        # FP16 iterations: the FP16-rounded dot may differ by one FP16 ulp (tensor-core
        # and NumPy FP32 sums differ in order and rounding before the FP16 rounding)
        sq = float(np.max(np.sum(X.astype(np.float64) ** 2, axis=1)))
        ulp = 2.0 ** (np.floor(np.log2(sq)) - 10)
        d2_err = np.abs(dist[same] ** 2 - od[same] ** 2)
        assert np.all(d2_err <= 2.5 * ulp + 1e-3 * od[same] ** 2), d2_err.max()
        if t >= 5:  # FP32 after the recompute; rows a converging 5th iteration left alone keep
            # FP16-era values, as the reference does, so a few entries carry the FP16 bound only
            close = np.isclose(dist[same], od[same], rtol=1e-4, atol=1e-4)
            assert close.mean() > 0.999, close.mean()
    # final quality equals the reference's
    ri, _ = oknn.knn_exact_f64(X, 15)
    assert abs(recall(idx, ri) - recall(g[f"idx_it{its[-1]}"].astype(np.int32), ri)) < 0.01


def test_nndescent_reverse_candidates_match_oracle():
    import torch

    from mlx_vis_b200 import _lib

    rng = np.random.default_rng(0)
    n, k = 500, 15
    idx = rng.integers(0, n, size=(n, k)).astype(np.int32)  # duplicates within rows on purpose
    want = onnd.reverse_candidates(idx)
    d_idx = torch.from_numpy(idx).cuda()
    rev = torch.empty_like(d_idx)
    ws = _lib.workspace(_lib.query("umapb_nnd_reverse_workspace", n, k), d_idx.device)
    _lib.call("umapb_nnd_reverse", _lib.ptr(d_idx), n, k, _lib.ptr(rev), _lib.ptr(ws), ws.numel(),
              _lib.stream_handle())
    assert np.array_equal(rev.cpu().numpy(), want)


@pytest.mark.parametrize("n,k", [(1003, 15), (37, 5), (2, 1)])
def test_nndescent_reverse_candidates_ragged_rows_and_hubs(n, k):
    """The reverse-bucket select works on groups of 4 rows: a last group with fewer
    rows and groups that mix buckets of more than 32 entries (hubs) with short ones."""
    import torch

    from mlx_vis_b200 import _lib

    rng = np.random.default_rng(n + k)
    idx = rng.integers(0, n, size=(n, k)).astype(np.int32)
    hubs = min(3, n - 1) + 1
    idx[: n // 2, 0] = rng.integers(0, hubs, size=n // 2)  # rows 0..hubs-1 become hubs
    want = onnd.reverse_candidates(idx)
    d_idx = torch.from_numpy(idx).cuda()
    rev = torch.full_like(d_idx, -7)
    ws = _lib.workspace(_lib.query("umapb_nnd_reverse_workspace", n, k), d_idx.device)
    _lib.call("umapb_nnd_reverse", _lib.ptr(d_idx), n, k, _lib.ptr(rev), _lib.ptr(ws), ws.numel(),
              _lib.stream_handle())
    got = rev.cpu().numpy()
    assert np.array_equal(got, want)


def test_nndescent_small_and_edge_cases():
    from mlx_vis_b200 import NNDescent

    rng = np.random.default_rng(3)
    for n, d, k in [(2, 3, 15), (17, 5, 15), (200, 130, 10), (1000, 100, 15)]:
        X = rng.normal(size=(n, d)).astype(np.float32)
        idx, dist = NNDescent(k=k, random_state=0).build(X)
        kk = min(k, n - 1)
        assert idx.shape == (n, kk) and dist.shape == (n, kk)
        assert np.all(idx != np.arange(n)[:, None])
        assert np.all(np.isfinite(dist)) and np.all(np.diff(dist, axis=1) >= -1e-3)
        if n <= 200:
            ri, _ = oknn.knn_exact_f64(X, kk)
            assert recall(idx, ri) > 0.9


def test_umap_with_nndescent(gauss2000):
    from sklearn.manifold import trustworthiness

    from mlx_vis_b200 import UMAP

    Y = UMAP(n_epochs=200, knn_method="nndescent", random_state=0).fit_transform(gauss2000)
    assert trustworthiness(gauss2000, Y, n_neighbors=15) > 0.95


@pytest.mark.parametrize("parallel", [True, False])
@pytest.mark.parametrize("n,k,d,seed", [(70000, 15, 784, 0), (5000, 15, 784, 3), (1000, 10, 150, 7), (257, 4, 64, 1),
                                        (2, 1, 5, 2), (3000, 32, 301, 11)])
def test_device_random_start_equals_numpy(n, k, d, seed, parallel):
    """umapb_nnd_random_start (grid-wide path and one-CTA walk) reproduces the
    reference's NumPy draws bit for bit and leaves NumPy's stream in the same state."""
    from mlx_vis_b200._nndescent.nndescent import random_start, random_start_device, words_state

    idx_h, P_h, P2_h = random_start(n, k, d, seed)
    st_h = np.random.get_state()
    idx, P, P2, state = random_start_device(n, k, d, seed, torch.device("cuda"), parallel=parallel)
    st = words_state(state.cpu().numpy())
    assert np.array_equal(idx.cpu().numpy(), idx_h)
    for got, want in ((P, P_h), (P2, P2_h)):
        assert (got is None) == (want is None)
        if got is not None:
            assert np.array_equal(got.cpu().numpy(), want)
    assert np.array_equal(st[1], st_h[1]) and st[2:] == st_h[2:]


@pytest.mark.parametrize("parallel", [True, False])
def test_device_random_start_continues_an_unseeded_stream(parallel):
    """random_state=None: the draws continue NumPy's global stream, including a
    cached second normal (has_gauss) and a mid-generation position."""
    from mlx_vis_b200._nndescent.nndescent import random_start, random_start_device, words_state

    np.random.seed(5)
    np.random.randn(3)  # leaves a cached normal
    np.random.randint(0, 10, 7)
    st0 = np.random.get_state()
    assert st0[3] == 1
    idx_h, P_h, P2_h = random_start(900, 6, 350, None)
    st_h = np.random.get_state()
    np.random.set_state(st0)
    idx, P, P2, state = random_start_device(900, 6, 350, None, torch.device("cuda"), parallel=parallel)
    st = words_state(state.cpu().numpy())
    assert np.array_equal(idx.cpu().numpy(), idx_h)
    assert np.array_equal(P.cpu().numpy(), P_h) and np.array_equal(P2.cpu().numpy(), P2_h)
    assert np.array_equal(st[1], st_h[1]) and st[2:] == st_h[2:]


def test_build_leaves_numpy_stream_like_the_reference():
    from mlx_vis_b200 import NNDescent
    from mlx_vis_b200._nndescent.nndescent import random_start

    X = np.random.default_rng(0).normal(size=(600, 40)).astype(np.float32)
    NNDescent(k=8, random_state=4).build(X)
    after = np.random.get_state()
    random_start(600, 8, 40, 4)
    want = np.random.get_state()
    assert np.array_equal(after[1], want[1]) and after[2:] == want[2:]


@pytest.mark.parametrize("half", [False, True])
@pytest.mark.parametrize("n,d,k,mc,j_nn", [(3000, 64, 15, 15, 15), (1000, 784, 15, 9, 7), (517, 36, 32, 20, 32),
                                           (40, 8, 5, 3, 2), (333, 12, 6, 6, 4), (700, 40, 33 - 1, 32, 16)])
def test_join_block_distances(n, d, k, mc, j_nn, half):
    """umapb_nnd_join: nnbuf[i][p*j_nn + j] = d(i, idx[idx[i][p]][j]) and curd[i][p] =
    d(i, idx[i][p]) with the iteration's distance rule (FP16 dots rounded to FP16)."""
    from mlx_vis_b200 import _lib

    rng = np.random.default_rng(n + d + k)
    X = rng.normal(size=(n, d)).astype(np.float32)
    idx = rng.integers(0, n - 1, size=(n, k)).astype(np.int32)
    idx = np.where(idx >= np.arange(n)[:, None], idx + 1, idx).astype(np.int32)
    Xd = torch.from_numpy(X).cuda()
    sq = torch.empty(n, dtype=torch.float32, device="cuda")
    s = _lib.stream_handle()
    _lib.call("umapb_nnd_sqnorms", _lib.ptr(Xd), n, d, 0, _lib.ptr(sq), s)
    if half:
        ldx = (d + 7) // 8 * 8
        src = torch.zeros((n, ldx), dtype=torch.float16, device="cuda")
        _lib.call("umapb_nnd_to_half", _lib.ptr(Xd), n, d, ldx, _lib.ptr(src), s)
        Xv = src[:, :d].float().cpu().numpy().astype(np.float64)
    else:
        ldx, src, Xv = d, Xd, X.astype(np.float64)
    d_idx = torch.from_numpy(idx).cuda()
    nnbuf = torch.full((n, mc * j_nn), -1.0, dtype=torch.float32, device="cuda")
    curd = torch.full((n, k), -1.0, dtype=torch.float32, device="cuda")
    evals = torch.zeros(1, dtype=torch.int64, device="cuda")
    ws = _lib.workspace(_lib.query("umapb_nnd_join_workspace", n, k, mc), Xd.device)
    # sources taken in a shuffled order: a scheduling choice that changes no output
    order = torch.from_numpy(rng.permutation(n).astype(np.int32)).cuda() if n % 2 else None
    # with mc == k the join's buckets also give the reverse candidates
    rev = torch.full((n, k), -7, dtype=torch.int32, device="cuda") if mc == k else None
    _lib.call("umapb_nnd_join", _lib.ptr(src), _lib.ptr(sq), d, ldx, int(half), _lib.ptr(d_idx), _lib.ptr(order), n,
              k, mc, j_nn, _lib.ptr(nnbuf), _lib.ptr(curd), _lib.ptr(rev), _lib.ptr(evals), _lib.ptr(ws), ws.numel(),
              s)
    if rev is not None:
        assert np.array_equal(rev.cpu().numpy(), onnd.reverse_candidates(idx))
    got_nn, got_cur = nnbuf.cpu().numpy(), curd.cpu().numpy()
    assert int(evals.item()) == n * mc * (1 + j_nn)
    sqh = sq.cpu().numpy().astype(np.float64)

    def want(i, c):
        dot = np.sum(Xv[i] * Xv[c], axis=-1)
        if half:
            dot = dot.astype(np.float32).astype(np.float16).astype(np.float64)
        return np.maximum(sqh[i] + sqh[c] - 2.0 * dot, 0.0), dot

    rows = np.repeat(np.arange(n), mc)
    srcs = idx[:, :mc].reshape(-1)
    w, dot = want(rows, srcs)
    # FP32 dot sums differ in order; FP16 rounding may then move one FP16 ulp
    tol = 1e-4 * (sqh[rows] + sqh[srcs]) + (2.5 * np.abs(dot) * 2.0 ** -10 if half else 0.0) + 1e-4
    assert np.all(np.abs(got_cur[:, :mc].reshape(-1) - w) <= tol)
    assert np.all(got_cur[:, mc:] == -1.0)  # positions >= mc are not written
    if j_nn:
        rr = np.repeat(rows, j_nn)
        cc = idx[np.repeat(srcs, j_nn), np.tile(np.arange(j_nn), len(srcs))]
        w2, dot2 = want(rr, cc)
        tol2 = 1e-4 * (sqh[rr] + sqh[cc]) + (2.5 * np.abs(dot2) * 2.0 ** -10 if half else 0.0) + 1e-4
        assert np.all(np.abs(got_nn.reshape(-1) - w2) <= tol2)


@pytest.mark.parametrize("n,d,k,mc,j_nn", [(3000, 64, 15, 3, 7), (1000, 784, 15, 9, 15), (517, 36, 32, 20, 32),
                                           (40, 8, 5, 3, 2)])
def test_join_new_sources(n, d, k, mc, j_nn):
    """umapb_nnd_join_new (converging path, nndescent.py:103-126): the sources of row i
    are its first mc neighbours in NEW-first stable order, and nnbuf[i][p*j_nn + j] =
    d(i, idx[s_p][j]) in FP32; rows without a NEW flag are left alone."""
    from mlx_vis_b200 import _lib

    rng = np.random.default_rng(n + d + k + mc)
    X = rng.normal(size=(n, d)).astype(np.float32)
    idx = rng.integers(0, n - 1, size=(n, k)).astype(np.int32)
    idx = np.where(idx >= np.arange(n)[:, None], idx + 1, idx).astype(np.int32)
    flags = (rng.random((n, k)) < 0.15).astype(np.uint8)
    flags[: n // 4] = 0  # a quarter of the rows have no NEW neighbour
    Xd = torch.from_numpy(X).cuda()
    sq = torch.empty(n, dtype=torch.float32, device="cuda")
    s = _lib.stream_handle()
    _lib.call("umapb_nnd_sqnorms", _lib.ptr(Xd), n, d, 0, _lib.ptr(sq), s)
    nnbuf = torch.full((n, mc * j_nn), -1.0, dtype=torch.float32, device="cuda")
    evals = torch.zeros(1, dtype=torch.int64, device="cuda")
    ws = _lib.workspace(_lib.query("umapb_nnd_join_workspace", n, k, k), Xd.device)
    order = torch.from_numpy(rng.permutation(n).astype(np.int32)).cuda() if n % 2 else None
    d_idx, d_flags = torch.from_numpy(idx).cuda(), torch.from_numpy(flags).cuda()  # alive until the sync below
    _lib.call("umapb_nnd_join_new", _lib.ptr(Xd), _lib.ptr(sq), d, _lib.ptr(d_idx), _lib.ptr(d_flags), _lib.ptr(order),
              n, k, mc, j_nn, _lib.ptr(nnbuf), _lib.ptr(evals), _lib.ptr(ws), ws.numel(), s)
    got = nnbuf.cpu().numpy()
    X64 = X.astype(np.float64)
    sqh = sq.cpu().numpy().astype(np.float64)
    active = flags.any(1)
    assert np.all(got[~active] == -1.0)
    assert int(evals.item()) == int(active.sum()) * mc * (1 + j_nn)
    for i in np.nonzero(active)[0][:300]:
        newf = np.nonzero(flags[i])[0]
        oldf = np.nonzero(flags[i] == 0)[0]
        srcs = idx[i, np.concatenate([newf, oldf])][:mc]
        cols = idx[np.repeat(srcs, j_nn), np.tile(np.arange(j_nn), mc)]
        want = np.maximum(sqh[i] + sqh[cols] - 2.0 * (X64[cols] @ X64[i]), 0.0)
        assert np.all(np.abs(got[i] - want) <= 1e-4 * (sqh[i] + sqh[cols]) + 1e-4)


@pytest.mark.parametrize("name,gen", [("gauss", ("gaussian_mixture", 3000, 32, 2)),
                                      ("proto", ("prototype_mixture", 2000, 784, 3))])
def test_join_and_row_kernel_builds_agree(name, gen, monkeypatch):
    """The blocked join changes where the nn-of-nn distances are computed, not the
    candidates or the rule: the graphs of both builds agree up to FP32 summation order."""
    from mlx_vis_b200 import NNDescent, datasets

    X = getattr(datasets, gen[0])(gen[1], gen[2], seed=gen[3])
    out = {}
    for on in ("1", "0"):
        monkeypatch.setenv("UMAPB_NND_JOIN", on)
        nn = NNDescent(k=15, random_state=42)
        idx, dist = nn.build(X)
        out[on] = (idx, dist, [h["changed"] for h in nn.history_], [h.get("join") for h in nn.history_])
    assert any(out["1"][3]) and not any(out["0"][3])
    assert recall(out["1"][0], out["0"][0]) > 0.995
    np.testing.assert_allclose(out["1"][2], out["0"][2], rtol=0.02, atol=20)
    same = out["1"][0] == out["0"][0]
    np.testing.assert_allclose(out["1"][1][same], out["0"][1][same], rtol=1e-3, atol=1e-3)


@pytest.mark.parametrize("k,gen", [(40, ("gaussian_mixture", 3000, 32, 2)), (91, ("gaussian_mixture", 2500, 16, 5)),
                                   (50, ("prototype_mixture", 2000, 784, 3))])
def test_nndescent_large_k_tracks_oracle(k, gen):
    """k above 32 (one block per row, every candidate distance in the row kernel;
    nnd_wide.cu): the same random start and iteration rules as the oracle, so the
    per-iteration update counts and the final graph follow it; the reference itself
    is calibrated at k = 91 (nndescent.py:85-88)."""
    from mlx_vis_b200 import NNDescent, datasets

    X = getattr(datasets, gen[0])(gen[1], gen[2], seed=gen[3])
    nn = NNDescent(k=k, random_state=42)
    idx, dist = nn.build(X)
    (oidx, odist), log = onnd.build(X, k=k, random_state=42, history=True)
    ours = np.array([h["changed"] for h in nn.history_])
    ref = np.array([l["changed"] for l in log])
    assert len(ours) == len(ref), (ours, ref)
    np.testing.assert_allclose(ours, ref, rtol=0.02, atol=20)
    overlap = np.mean([len(set(a) & set(b)) / k for a, b in zip(idx, oidx)])
    assert overlap > 0.99, overlap
    assert np.all(idx != np.arange(len(X))[:, None])
    assert all(len(set(r)) == k for r in idx)
    assert np.all(np.diff(dist, axis=1) >= 0)
    ri, _ = oknn.knn_exact_f64(X, k)
    assert abs(recall(idx, ri) - recall(oidx, ri)) < 0.01


def test_umap_with_fifty_neighbours(gauss2000):
    """UMAP(n_neighbors=50, knn_method="nndescent") runs end to end (the reference
    has no limit on k)."""
    from sklearn.manifold import trustworthiness

    from mlx_vis_b200 import UMAP

    Y = UMAP(n_neighbors=50, n_epochs=100, knn_method="nndescent", random_state=0).fit_transform(gauss2000)
    assert Y.shape == (2000, 2) and np.isfinite(Y).all()
    assert trustworthiness(gauss2000, Y, n_neighbors=15) > 0.93


def test_nndescent_k_above_the_envelope_is_rejected():
    from mlx_vis_b200 import NNDescent

    with pytest.raises(ValueError, match="k <= 100"):
        NNDescent(k=101).build(np.zeros((200, 4), dtype=np.float32))


@pytest.mark.parametrize("n,d,k,blocks", [(3001, 64, 15, 8), (1000, 36, 32, 3), (257, 784, 5, 1), (500, 20, 10, 7)])
def test_pair_gathers_by_row_block_equal_the_gather(n, d, k, blocks):
    """umapb_nnd_gather_pairs once per row block (the pairs whose later row is in it)
    and then umapb_nnd_sort_rows give exactly what the one-shot gather with its row sort
    gives: the same pair values, bit for bit, and the same order."""
    from mlx_vis_b200 import _lib

    rng = np.random.default_rng(n + k)
    X = torch.from_numpy(rng.standard_normal((n, d)).astype(np.float32)).cuda()
    idx0 = rng.integers(0, n, (n, k)).astype(np.int32)
    idx0[0, :] = 0  # a row that lists itself
    idx0[1, : k // 2] = 7  # repeated neighbours
    s = _lib.stream_handle()
    sq = torch.empty(n, dtype=torch.float32, device="cuda")
    _lib.call("umapb_nnd_sqnorms", _lib.ptr(X), n, d, 0, _lib.ptr(sq), s)
    ia = torch.from_numpy(idx0).cuda()
    da = torch.full((n, k), -1.0, device="cuda")
    _lib.call("umapb_nnd_gather", _lib.ptr(X), _lib.ptr(sq), n, d, _lib.ptr(ia), _lib.ptr(da), k, 1, s)
    ib = torch.from_numpy(idx0).cuda()
    db = torch.full((n, k), -1.0, device="cuda")
    cuts = np.linspace(0, n, blocks + 1).astype(int)
    cuts[1:-1] += rng.integers(-3, 4, blocks - 1)  # uneven blocks
    for r0, r1 in zip(cuts[:-1], cuts[1:]):
        _lib.call("umapb_nnd_gather_pairs", _lib.ptr(X), _lib.ptr(sq), n, d, _lib.ptr(ib), _lib.ptr(db), k,
                  int(r0), int(r1), s)
    assert bool((db >= 0).all())  # every pair was computed once the last block arrived
    _lib.call("umapb_nnd_sort_rows", _lib.ptr(ib), _lib.ptr(db), n, k, s)
    assert np.array_equal(ia.cpu().numpy(), ib.cpu().numpy())
    assert np.array_equal(da.cpu().numpy().view(np.int32), db.cpu().numpy().view(np.int32))
