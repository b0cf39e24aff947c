"""Generate ``tests/golden/pca_proto.npz``: the PCA preprocessing of the REFERENCE
``UMAP.fit_transform`` (hanxiao/mlx-vis 0.7.0, mlx_vis/_umap/umap.py:92-113), run
unmodified on CPU with ``oracle/mlx_shim`` standing in for ``mlx``.

The reference hands the projected data to ``compute_knn`` (umap.py:117-121); the
script wraps that function to record its input and stop the fit there, so the
fixture holds exactly the reference's ``X_for_knn`` for
``prototype_mixture(1000, 784, seed=4)`` with ``pca_dim=20``.

Usage (needs the reference checkout; it is NOT needed to run the tests):

    MLX_VIS_REFERENCE=/path/to/mlx-vis python tests/golden/make_golden_pca.py
"""

from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

from make_golden import _load_reference, sha  # noqa: E402


class _Captured(Exception):
    pass


def main():
    mx, ref_knn, ref_nnd, ref_umap = _load_reference()
    from mlx_vis_b200.datasets import prototype_mixture

    X = prototype_mixture(1000, 784, seed=4)
    seen = {}

    def capture(X_for_knn, *args, **kwargs):
        seen["X"] = np.array(X_for_knn, dtype=np.float32)
        raise _Captured()

    ref_knn.compute_knn = capture  # fit_transform imports it from the module at call time
    u = ref_umap.UMAP(n_components=2, pca_dim=20, random_state=0)
    try:
        u.fit_transform(X)
    except _Captured:
        pass
    Xp = seen["X"]
    assert Xp.shape == (1000, 20)
    np.savez_compressed(os.path.join(HERE, "pca_proto.npz"), X_pca=Xp)
    mpath = os.path.join(HERE, "manifest.json")
    with open(mpath) as f:
        manifest = json.load(f)
    manifest["fixtures"]["pca_proto"] = {"gen": "prototype_mixture(1000, 784, seed=4)", "sha": sha(X),
                                         "pca_dim": 20,
                                         "note": "X_for_knn of UMAP.fit_transform (umap.py:92-113)"}
    with open(mpath, "w") as f:
        json.dump(manifest, f, indent=1, sort_keys=True)
    print("wrote pca_proto", Xp.shape)


if __name__ == "__main__":
    main()
