"""Generate the 70,000 x 784 fixture (``tests/golden/c3_70k.npz``) by running the
REFERENCE implementation (hanxiao/mlx-vis 0.7.0) unmodified on CPU, with
``oracle/mlx_shim`` standing in for the ``mlx`` package that cannot be installed
offline.  This is the workload the benchmark times: ``prototype_mixture(70000,
784, seed=0)``, ``UMAP(n_components=2, n_neighbors=15, min_dist=0.1,
n_epochs=500, knn_method="nndescent", random_state=0)``.

The stages are called in the order of ``UMAP.fit_transform`` (umap.py:117-144)
so that each one can be timed; the result equals ``fit_transform``'s.

Stored (the tests regenerate X from the generator and check its SHA-256):

* ``idx``            the reference's NNDescent graph (70000, 15) int32
                     (nndescent.py:34-403 through _knn.py:35-45)
* ``updates``        its per-iteration update counts (verbose log)
* ``sample``         10,000 fixed rows (rng 0) on which trustworthiness@15 is taken
* ``embedding_sample`` the reference embedding on those rows
* ``exact_rows`` / ``exact_idx``  exact float64 kNN (k=15, self excluded) of 2,000
                     fixed rows (rng 1) against all 70,000, for recall
* meta: trustworthiness@15 on the sample, recall of the reference graph on the
  exact rows, edge count, positive-edge updates, per-stage CPU seconds

Usage (needs the reference checkout; it is NOT needed to run the tests):

    MLX_VIS_REFERENCE=/path/to/mlx-vis python tests/golden/make_golden_70k.py

Runs for tens of minutes on 8 cores (the reference's NumPy-backed NNDescent and
500 layout epochs dominate).
"""

from __future__ import annotations

import contextlib
import io
import json
import os
import re
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

from make_golden import REPO, _load_reference, sha  # noqa: E402

N, D, K, EPOCHS = 70000, 784, 15, 500


def exact_rows_knn(X: np.ndarray, rows: np.ndarray, k: int, chunk: int = 250) -> np.ndarray:
    """Exact float64 kNN of ``rows`` against all of X (self excluded; ties by index)."""
    X64 = X.astype(np.float64)
    sq = np.einsum("ij,ij->i", X64, X64)
    out = np.empty((len(rows), k), dtype=np.int32)
    for s in range(0, len(rows), chunk):
        r = rows[s:s + chunk]
        d2 = sq[r][:, None] + sq[None, :] - 2.0 * (X64[r] @ X64.T)
        d2[np.arange(len(r)), r] = np.inf
        part = np.argpartition(d2, k, axis=1)[:, :k + 1]
        for j, i in enumerate(r):
            cand = part[j]
            order = np.lexsort((cand, d2[j, cand]))
            out[s + j] = cand[order][:k]
    return out


def main():
    mx, ref_knn, ref_nnd, ref_umap = _load_reference()
    from mlx_vis_b200.datasets import prototype_mixture
    from sklearn.manifold import trustworthiness

    X = prototype_mixture(N, D, seed=0)
    u = ref_umap.UMAP(n_components=2, n_neighbors=K, min_dist=0.1, n_epochs=EPOCHS, knn_method="nndescent",
                      random_state=0)
    times = {}
    t = time.perf_counter()
    buf = io.StringIO()
    with contextlib.redirect_stdout(buf):
        # fit_transform's kNN call (umap.py:117-121) with the verbose log for the update counts
        nn = ref_nnd.NNDescent(k=K, verbose=True, random_state=0)
        idx, dist = nn.build(X)
    times["knn"] = time.perf_counter() - t
    updates = [int(m) for m in re.findall(r"Iter \d+/\d+: (\d+) updates", buf.getvalue())]
    print("NNDescent", times["knn"], "s; updates", updates, flush=True)

    t = time.perf_counter()
    rows, cols, vals = u._fuzzy_simplicial_set(idx, dist, N)
    mx.eval(rows, cols, vals)
    times["fuzzy"] = time.perf_counter() - t
    a, b = u._find_ab_params(u.spread, u.min_dist)
    t = time.perf_counter()
    mx.random.seed(0)
    Y = u._spectral_init(rows, cols, vals, N)
    mx.eval(Y)
    times["init"] = time.perf_counter() - t
    print("fuzzy", times["fuzzy"], "init", times["init"], flush=True)
    t = time.perf_counter()
    Y = np.array(u._optimize(rows, cols, vals, Y, a, b, N))
    times["layout"] = time.perf_counter() - t
    print("layout", times["layout"], flush=True)

    w = np.array(vals).astype(np.float32)
    n_samples = EPOCHS * (w / float(w.max()))
    eps = np.where(n_samples > 0, EPOCHS / n_samples, -1.0).astype(np.float32)
    nxt = eps.copy()
    edge_updates = 0
    for e in range(EPOCHS):
        act = nxt <= e
        c = int(act.sum())
        if c:
            nxt[act] += eps[act]
            edge_updates += c

    sample = np.sort(np.random.default_rng(0).choice(N, 10000, replace=False)).astype(np.int32)
    tw = float(trustworthiness(X[sample], Y[sample], n_neighbors=15))
    exact_rows = np.sort(np.random.default_rng(1).choice(N, 2000, replace=False)).astype(np.int32)
    exact_idx = exact_rows_knn(X, exact_rows, K)
    ref_recall = float(np.mean([len(set(a) & set(b)) / K for a, b in zip(idx[exact_rows], exact_idx)]))
    print("trustworthiness", tw, "recall", ref_recall, flush=True)

    meta = {"gen": f"prototype_mixture({N}, {D}, seed=0)", "sha": sha(X),
            "umap": {"n_components": 2, "n_neighbors": K, "min_dist": 0.1, "n_epochs": EPOCHS,
                     "knn_method": "nndescent", "random_state": 0},
            "trustworthiness15_sample": tw, "nnd_recall_exact_rows": ref_recall,
            "n_edges": int(np.array(rows).shape[0]), "edge_updates": edge_updates,
            "cpu_stage_s": {k: round(v, 2) for k, v in times.items()},
            "cpu_fit_s": round(sum(times.values()), 2), "cpu_threads": os.cpu_count(),
            "cpu_note": "reference code on the NumPy mlx shim, one process, NumPy's own threading"}
    np.savez_compressed(os.path.join(HERE, "c3_70k.npz"), idx=idx.astype(np.int32),
                        updates=np.asarray(updates, dtype=np.int64), sample=sample,
                        embedding_sample=Y[sample].astype(np.float32), exact_rows=exact_rows, exact_idx=exact_idx)
    mpath = os.path.join(HERE, "manifest.json")
    with open(mpath) as f:
        manifest = json.load(f)
    manifest["fixtures"]["c3_70k"] = meta
    with open(mpath, "w") as f:
        json.dump(manifest, f, indent=1, sort_keys=True)
    print(json.dumps(meta, indent=1))


if __name__ == "__main__":
    main()
