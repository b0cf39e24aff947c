"""Generate the golden fixtures under tests/golden/ by running the REFERENCE
implementation (hanxiao/mlx-vis 0.7.0: ``mlx_vis/_knn.py``,
``mlx_vis/_nndescent/nndescent.py``, ``mlx_vis/_umap/umap.py``) unmodified on
CPU, with ``oracle/mlx_shim`` standing in for the ``mlx`` package that cannot be
installed offline.

Usage (needs the reference checkout; it is NOT needed to run the tests):

    MLX_VIS_REFERENCE=/path/to/mlx-vis python tests/golden/make_golden.py

The reference package's ``__init__`` imports every method and the plotting
layer, so only the three hot-path modules are loaded, through namespace stubs.
Inputs are regenerated in the tests from ``mlx_vis_b200.datasets`` with the
seeds stored here; a SHA-256 of each input is stored to catch generator drift.
"""

from __future__ import annotations

import contextlib
import hashlib
import io
import json
import os
import re
import sys
import types

import warnings

import numpy as np

warnings.simplefilter("ignore", RuntimeWarning)

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REF = os.environ.get("MLX_VIS_REFERENCE")

sys.path.insert(0, os.path.join(REPO, "oracle", "mlx_shim"))
sys.path.insert(0, REPO)


def _load_reference():
    if not REF or not os.path.isdir(os.path.join(REF, "mlx_vis")):
        raise SystemExit("set MLX_VIS_REFERENCE to a checkout of hanxiao/mlx-vis (the directory holding mlx_vis/)")
    for name, sub in [("mlx_vis", "mlx_vis"), ("mlx_vis._umap", "mlx_vis/_umap"),
                      ("mlx_vis._nndescent", "mlx_vis/_nndescent")]:
        mod = types.ModuleType(name)
        mod.__path__ = [os.path.join(REF, sub)]
        sys.modules[name] = mod
    import mlx.core as mx  # the shim
    import mlx_vis._knn as ref_knn
    import mlx_vis._nndescent.nndescent as ref_nnd
    import mlx_vis._umap.umap as ref_umap
    return mx, ref_knn, ref_nnd, ref_umap


def sha(x: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(x).tobytes()).hexdigest()[:16]


def nnd_with_log(ref_nnd, X, **kw):
    buf = io.StringIO()
    nn = ref_nnd.NNDescent(verbose=True, **kw)
    with contextlib.redirect_stdout(buf):
        idx, dist = nn.build(X)
    updates = [int(m) for m in re.findall(r"Iter \d+/\d+: (\d+) updates", buf.getvalue())]
    return idx, dist, np.asarray(updates, dtype=np.int64)


def main():
    mx, ref_knn, ref_nnd, ref_umap = _load_reference()
    from mlx_vis_b200.datasets import gaussian_mixture, prototype_mixture
    from sklearn.manifold import trustworthiness

    manifest = {"reference": "hanxiao/mlx-vis 0.7.0 (run on oracle/mlx_shim)", "fixtures": {}}

    def save(name, meta, **arrays):
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrays)
        manifest["fixtures"][name] = meta
        print("wrote", name, {k: (v.shape, str(v.dtype)) for k, v in arrays.items()})

    # 1. brute kNN (_knn.py:47-88) on the 2000x64 Gaussian mixture and a 1500x784 prototype mixture
    X1 = gaussian_mixture(2000, 64, seed=0)
    i1, d1 = ref_knn.compute_knn(X1, 15, method="brute")
    save("knn_brute_gauss", {"gen": "gaussian_mixture(2000, 64, seed=0)", "sha": sha(X1), "k": 15},
         idx=i1.astype(np.int32), dist=d1.astype(np.float32))
    Xp = prototype_mixture(1500, 784, seed=1)
    ip, dp = ref_knn.compute_knn(Xp, 15, method="brute")
    save("knn_brute_proto", {"gen": "prototype_mixture(1500, 784, seed=1)", "sha": sha(Xp), "k": 15},
         idx=ip.astype(np.int32), dist=dp.astype(np.float32))

    # 2. NNDescent (nndescent.py:34-403): full-dimension path and the projection path (d > 100)
    Xn = gaussian_mixture(3000, 32, seed=2)
    res = {}
    for t in (1, 2, 3, 20):
        idx, dist, upd = nnd_with_log(ref_nnd, Xn, k=15, random_state=42, n_iters=t)
        res[f"idx_it{t}"] = idx.astype(np.int32)
        res[f"dist_it{t}"] = dist.astype(np.float32)
        res[f"updates_it{t}"] = upd
    save("nnd_gauss", {"gen": "gaussian_mixture(3000, 32, seed=2)", "sha": sha(Xn), "k": 15,
                       "random_state": 42}, **res)

    Xq = prototype_mixture(2000, 784, seed=3)
    res = {}
    for t in (1, 2, 5, 20):
        idx, dist, upd = nnd_with_log(ref_nnd, Xq, k=15, random_state=42, n_iters=t)
        res[f"idx_it{t}"] = idx.astype(np.int16)
        res[f"dist_it{t}"] = dist.astype(np.float32)
        res[f"updates_it{t}"] = upd
    save("nnd_proto", {"gen": "prototype_mixture(2000, 784, seed=3)", "sha": sha(Xq), "k": 15,
                       "random_state": 42}, **res)

    # 3. fuzzy simplicial set (umap.py:199-270) on the brute graph of (1), n_epochs=200
    u = ref_umap.UMAP(n_neighbors=15, min_dist=0.1, n_epochs=200, random_state=0)
    rows, cols, vals = u._fuzzy_simplicial_set(i1, d1, X1.shape[0])
    rows, cols, vals = np.array(rows), np.array(cols), np.array(vals)
    save("fuzzy_gauss", {"from": "knn_brute_gauss", "n_epochs": 200, "k": 15},
         rows=rows.astype(np.int32), cols=cols.astype(np.int32), vals=vals.astype(np.float32))

    # fuzzy set edge cases: duplicated points (zero distances), k=5, n_epochs=500
    rng = np.random.default_rng(7)
    Xd = rng.standard_normal((300, 8)).astype(np.float32)
    Xd[100:130] = Xd[0:30]          # exact duplicates -> zero kNN distances
    Xd[200:203] = Xd[5]             # a point with three copies
    idd, ddd = ref_knn.compute_knn(Xd, 5, method="brute")
    u5 = ref_umap.UMAP(n_neighbors=5, n_epochs=500, random_state=0)
    r5, c5, v5 = u5._fuzzy_simplicial_set(idd, ddd, Xd.shape[0])
    save("fuzzy_dups", {"gen": "normal(300, 8) rng 7 with duplicated rows", "sha": sha(Xd), "k": 5,
                        "n_epochs": 500},
         X=Xd, knn_idx=idd.astype(np.int32), knn_dist=ddd.astype(np.float32),
         rows=np.array(r5).astype(np.int32), cols=np.array(c5).astype(np.int32),
         vals=np.array(v5).astype(np.float32))

    # 4. a, b curve fit (umap.py:272-296)
    grid = np.array([[1.0, 0.1], [1.0, 0.0], [1.0, 0.5], [2.0, 0.25], [0.5, 0.05], [1.0, 0.25],
                     [1.0, 0.8], [0.5, 0.1], [1.5, 0.3]])
    ab = np.array([ref_umap.UMAP._find_ab_params(s, m) for s, m in grid])
    # settings for which the reference's Gauss-Newton diverges and lstsq raises LinAlgError
    diverging = np.array([[1.0, 0.99], [3.0, 1.0]])
    for s, m in diverging:
        try:
            ref_umap.UMAP._find_ab_params(s, m)
            raise SystemExit(f"expected LinAlgError for spread={s}, min_dist={m}")
        except np.linalg.LinAlgError:
            pass
    save("ab_params", {"columns": ["spread", "min_dist"],
                       "diverging": "grid rows of `diverging` raise numpy.linalg.LinAlgError"},
         grid=grid, ab=ab, diverging=diverging)

    # 5. spectral init (umap.py:298-357) with the shim's seeded draws logged as V0
    mx.random.seed(0)
    mx.random.log.clear()
    Y0 = np.array(u._spectral_init(mx.array(rows), mx.array(cols), mx.array(vals), X1.shape[0]))
    V0 = mx.random.log[0][1]
    save("spectral_gauss", {"from": "fuzzy_gauss", "random_state": 0, "noise_seed": 42},
         V0=V0.astype(np.float32), Y0=Y0.astype(np.float32))

    # 6. optimize_layout (umap.py:389-449): snapshots + the negative samples of the first epochs
    a, b = ref_umap.UMAP._find_ab_params(1.0, 0.1)
    mx.random.seed(0)
    mx.random.log.clear()
    snaps = {}
    keep = {0, 1, 2, 3, 10, 50, 200}

    def cb(epoch, Y):
        if epoch in keep:
            snaps[epoch] = Y.copy()

    Yf = np.array(u._optimize(mx.array(rows), mx.array(cols), mx.array(vals), mx.array(Y0), a, b,
                              X1.shape[0], epoch_callback=cb))
    negs = [v for kind, v in mx.random.log if kind == "randint"]
    # active-set sizes per epoch from the reference's own host schedule (umap.py:401-414)
    w = vals.astype(np.float32)
    n_samples = 200 * (w / float(w.max()))
    eps = np.where(n_samples > 0, 200 / n_samples, -1.0)
    nxt = eps.copy()
    n_active = []
    for e in range(200):
        act = np.where(nxt <= e)[0]
        if len(act):
            nxt[act] += eps[act]
        n_active.append(len(act))
    arrays = {f"Y_ep{e}": snaps[e].astype(np.float32) for e in sorted(snaps)}
    for j in range(3):
        arrays[f"neg_{j}"] = negs[j].astype(np.int16)
    save("optimize_gauss", {"from": "spectral_gauss", "n_epochs": 200, "a": a, "b": b,
                            "learning_rate": 1.0, "negative_sample_rate": 5,
                            "neg_k": "neg_j holds the randint draw of the j-th non-empty epoch"},
         n_active=np.asarray(n_active, dtype=np.int32), Y_final=Yf.astype(np.float32), **arrays)

    # 7. full fit_transform on the 2000x64 workload (200 epochs, brute, seed 0)
    mx.random.seed(0)
    uf = ref_umap.UMAP(n_components=2, n_neighbors=15, min_dist=0.1, n_epochs=200,
                       knn_method="brute", random_state=0)
    Yu = uf.fit_transform(X1)
    tw = float(trustworthiness(X1, Yu, n_neighbors=15))
    save("umap_gauss", {"gen": "gaussian_mixture(2000, 64, seed=0)", "sha": sha(X1), "n_epochs": 200,
                        "trustworthiness15": tw},
         embedding=Yu.astype(np.float32))

    with open(os.path.join(HERE, "manifest.json"), "w") as f:
        json.dump(manifest, f, indent=1, sort_keys=True)
    print("trustworthiness@15 of the reference embedding:", tw)


if __name__ == "__main__":
    main()
