"""NNDescent oracle (test infrastructure): a NumPy restatement of the reference's
``NNDescent.build`` (mlx_vis/_nndescent/nndescent.py:34-403) and helpers.

Semantics fixed here where MLX leaves them open (and mirrored by the CUDA
kernels):  argsorts are stable, and the top-k of a candidate row keeps the k
smallest (distance, id) pairs in that order.  The random stream is the
reference's own: ``np.random.seed`` + ``randint`` + two ``randn`` projections
from NumPy's global MT19937, so the random init and projections are identical.
"""

from __future__ import annotations

import numpy as np

_BIG = np.float32(1e30)


def _chunk_rows(c: int, d: int) -> int:
    # rows per gather chunk: about 2^25 gathered values, so large k stays in memory;
    # every row's dot products are independent, so chunking changes no value
    return max(1, (1 << 25) // max(c * d, 1))


def gather_d2(Xd: np.ndarray, sq: np.ndarray, cols: np.ndarray) -> np.ndarray:
    """_gather_dists (nndescent.py:573-612): max(sq_i + sq_c - 2 x_i.x_c, 0), float32."""
    n, c = cols.shape
    out = np.empty((n, c), dtype=np.float32)
    step = _chunk_rows(c, Xd.shape[1])
    for s in range(0, n, step):
        e = min(s + step, n)
        flat = cols[s:e].reshape(-1)
        dots = np.einsum("id,icd->ic", Xd[s:e], Xd[flat].reshape(e - s, c, Xd.shape[1]))
        out[s:e] = np.maximum(sq[s:e, None] + sq[flat].reshape(e - s, c) - np.float32(2.0) * dots, np.float32(0))
    return out


def gather_d2_half(Xd: np.ndarray, sq: np.ndarray, cols: np.ndarray) -> np.ndarray:
    """_gather_dists_half (nndescent.py:615-641): float16 operands, the dot rounded to
    float16 (float32 accumulation), norms kept in float32."""
    n, c = cols.shape
    Xh = Xd.astype(np.float16).astype(np.float32)
    out = np.empty((n, c), dtype=np.float32)
    step = _chunk_rows(c, Xd.shape[1])
    for s in range(0, n, step):
        e = min(s + step, n)
        flat = cols[s:e].reshape(-1)
        dots = np.einsum("id,icd->ic", Xh[s:e], Xh[flat].reshape(e - s, c, Xd.shape[1]))
        dots = dots.astype(np.float16).astype(np.float32)
        out[s:e] = np.maximum(sq[s:e, None] + sq[flat].reshape(e - s, c) - np.float32(2.0) * dots, np.float32(0))
    return out


def reverse_candidates(indices: np.ndarray) -> np.ndarray:
    """_compute_reverse_candidates (nndescent.py:406-436): slot p of row j holds the
    p-th smallest source i with j in knn(i); slots beyond j's in-degree hold 0."""
    n, k = indices.shape
    src = np.repeat(np.arange(n, dtype=np.int32), k)
    dst = indices.reshape(-1)
    order = np.argsort(dst, kind="stable")
    rs, rd = src[order], dst[order]
    new_group = np.concatenate([[True], rd[1:] != rd[:-1]])
    pos = np.arange(n * k)
    start = np.maximum.accumulate(np.where(new_group, pos, 0))
    within = pos - start
    keep = within < k
    out = np.zeros(n * k, dtype=np.int32)
    out[rd[keep].astype(np.int64) * k + within[keep]] = rs[keep]
    return out.reshape(n, k)


def dedup_topk(cands: np.ndarray, d2: np.ndarray, k: int):
    """_dedup_topk_block (nndescent.py:439-458): sort by id, later duplicates -> 1e30,
    keep the k smallest (distance, id) pairs in ascending order."""
    o = np.argsort(cands, axis=1, kind="stable")
    sc = np.take_along_axis(cands, o, axis=1)
    sd = np.take_along_axis(d2, o, axis=1).copy()
    dup = np.zeros_like(sc, dtype=bool)
    dup[:, 1:] = sc[:, 1:] == sc[:, :-1]
    sd[dup] = _BIG
    sel = np.lexsort((sc, sd), axis=1)[:, :k]
    return np.take_along_axis(sc, sel, axis=1).astype(np.int32), np.take_along_axis(sd, sel, axis=1)


def iteration_params(update_frac: float, k: int, mc: int):
    """Per-iteration candidate counts (nndescent.py:100-101, 107, 223)."""
    mc_nn = max(3, int(min(k, mc) * min(1.0, update_frac ** 0.5 * 3)))
    j_nn = max(k // 2, min(k, int(k * min(1.0, update_frac ** 0.5 * 3))))
    mc_conv = max(3, int(k * update_frac))
    return mc_nn, j_nn, mc_conv


def random_init(n: int, k: int, d: int, random_state):
    """The reference's random draws, in order (nndescent.py:47-57, 72-82)."""
    if random_state is not None:
        np.random.seed(random_state)
    idx = np.random.randint(0, n - 1, (n, k), dtype=np.int32)
    i_vals = np.arange(n, dtype=np.int32)[:, None]
    idx = np.where(idx >= i_vals, idx + 1, idx).astype(np.int32)
    pd1, pd2 = min(100, d), min(300, d)
    P = (np.random.randn(d, pd1).astype(np.float32) / np.sqrt(pd1)).astype(np.float32) if pd1 < d else None
    P2 = (np.random.randn(d, pd2).astype(np.float32) / np.sqrt(pd2)).astype(np.float32) if pd2 < d else None
    return idx, P, P2


def build(X, k=15, n_iters=20, max_candidates=None, delta=0.015, random_state=None, history=False):
    """NNDescent.build (nndescent.py:34-403).  Returns (idx int32, dist float32 Euclidean)
    and, with ``history=True``, a list of per-iteration dicts."""
    X = np.ascontiguousarray(X, dtype=np.float32)
    n, d = X.shape
    k = min(k, n - 1)
    mc = max_candidates or k
    sq = np.sum(X * X, axis=1, dtype=np.float32)
    indices, P, P2 = random_init(n, k, d, random_state)
    dists = gather_d2(X, sq, indices)
    si = np.argsort(dists, axis=1, kind="stable")
    indices = np.take_along_axis(indices, si, axis=1)
    dists = np.take_along_axis(dists, si, axis=1)
    if P is not None:
        X_low = X @ P
        sq_low = np.sum(X_low * X_low, axis=1, dtype=np.float32)
    else:
        X_low, sq_low = X, sq

    log = []
    update_frac = 1.0
    flags = np.ones((n, k), dtype=bool)
    rows_all = np.arange(n, dtype=np.int32)
    for it in range(n_iters):
        mc_nn, j_nn, mc_conv = iteration_params(update_frac, k, mc)
        if update_frac < 0.5:
            # converging path (nndescent.py:103-220)
            new_order = np.argsort((~flags).astype(np.int32), axis=1, kind="stable")
            new_first = np.take_along_axis(indices, new_order, axis=1)
            mc_new = mc_conv
            active = np.nonzero(flags.any(axis=1))[0].astype(np.int32)
            use_rev = update_frac >= 0.10
            nn_sub = new_first[active, :mc_new]
            nc = indices[nn_sub.reshape(-1)].reshape(len(active), mc_new, k)[:, :, :j_nn]
            nc = nc.reshape(len(active), mc_new * j_nn)
            if use_rev:
                nc = np.concatenate([nc, reverse_candidates(indices)[active]], axis=1)
            new_d = np.empty(nc.shape, dtype=np.float32)
            step = _chunk_rows(nc.shape[1], d)
            for s in range(0, len(active), step):
                e = min(s + step, len(active))
                flat = nc[s:e].reshape(-1)
                dots = np.einsum("id,icd->ic", X[active[s:e]], X[flat].reshape(e - s, nc.shape[1], d))
                new_d[s:e] = np.maximum(sq[active[s:e], None] + sq[flat].reshape(e - s, nc.shape[1])
                                        - np.float32(2.0) * dots, np.float32(0))
            ac = np.concatenate([indices[active], nc], axis=1)
            ad = np.concatenate([dists[active], new_d], axis=1)
            ad = np.where(ac == active[:, None], _BIG, ad)
            ri, rd = dedup_topk(ac, ad, k)
            new_indices, new_dists = indices.copy(), dists.copy()
            new_indices[active] = ri
            new_dists[active] = rd
            info = dict(path="converging", mc_new=mc_new, j_nn=j_nn, use_rev=use_rev, n_active=len(active))
        else:
            # full path (nndescent.py:221-378)
            mc_new = mc_nn
            if it == 0:
                Xd, sq_d = X_low, sq_low
            elif it == 1 and P2 is not None:
                Xd = X @ P2
                sq_d = np.sum(Xd * Xd, axis=1, dtype=np.float32)
            else:
                Xd, sq_d = X, sq
            use_half = it in (1, 2, 3, 4)
            recompute_cur = (it == 0) or use_half
            use_rev = update_frac >= 0.10
            nn_sub = indices[:, :mc_new]
            nc = indices[nn_sub.reshape(-1)].reshape(n, mc_new, k)[:, :, :j_nn].reshape(n, mc_new * j_nn)
            if use_rev:
                nc = np.concatenate([nc, reverse_candidates(indices)], axis=1)
            g = gather_d2_half if use_half else gather_d2
            new_d = g(Xd, sq_d, nc)
            cur_d = g(Xd, sq_d, indices) if recompute_cur else dists
            ac = np.concatenate([indices, nc], axis=1)
            ad = np.concatenate([cur_d, new_d], axis=1)
            ad = np.where(ac == rows_all[:, None], _BIG, ad)
            new_indices, new_dists = dedup_topk(ac, ad, k)
            if it == 4:
                new_dists = gather_d2(X, sq, new_indices)
            info = dict(path="full", mc_new=mc_new, j_nn=j_nn, use_rev=use_rev, use_half=use_half,
                        space=int(Xd.shape[1]))
        flags = new_indices != indices
        changed = int(flags.sum())
        update_frac = changed / (n * k)
        indices, dists = new_indices, new_dists
        info.update(it=it, changed=changed)
        log.append(info)
        if update_frac < delta:
            break
    out = (indices, np.sqrt(np.maximum(dists, 0)).astype(np.float32))
    return (out, log) if history else out
