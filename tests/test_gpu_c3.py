"""The benchmark workload itself against the reference's own run on the same input.

70,000 x 784 seeded prototype mixture (10 classes), UMAP(n_components=2,
n_neighbors=15, min_dist=0.1, n_epochs=500, knn_method="nndescent",
random_state=0): the reference's NNDescent graph, its update log, its recall
against exact kNN on 2,000 fixed rows and its trustworthiness@15 on 10,000 fixed
rows come from tests/golden/c3_70k.npz (the reference's modules run unmodified
on the NumPy mlx shim by tests/golden/make_golden_70k.py).
"""

import hashlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def c3(golden, manifest):
    from mlx_vis_b200.datasets import prototype_mixture

    m = manifest["c3_70k"]
    X = prototype_mixture(70000, 784, seed=0)
    assert hashlib.sha256(X.tobytes()).hexdigest()[:16] == m["sha"]
    return X, golden("c3_70k"), m


def _row_overlap(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """|set(a_i) & set(b_i)| / k per row (rows hold distinct ids)."""
    return (a[:, :, None] == b[:, None, :]).any(axis=2).sum(axis=1) / a.shape[1]


def test_c3_nndescent_tracks_the_reference_build(c3):
    """Same random start (NumPy's stream, bit for bit), same iteration rules: the
    per-iteration update counts follow the reference's log, the graphs share most
    neighbours, and the recall against exact kNN equals the reference's within 0.01."""
    from mlx_vis_b200 import NNDescent

    X, g, m = c3
    nn = NNDescent(k=15, random_state=0)
    idx, dist = nn.build(X)
    ours = np.array([h["changed"] for h in nn.history_])
    ref = g["updates"]
    assert len(ours) == len(ref), (ours, ref)
    np.testing.assert_allclose(ours, ref, rtol=0.02)
    overlap = _row_overlap(idx, g["idx"]).mean()
    assert overlap > 0.95, overlap
    rows = g["exact_rows"]
    recall = _row_overlap(idx[rows], g["exact_idx"]).mean()
    assert abs(recall - m["nnd_recall_exact_rows"]) <= 0.01, (recall, m["nnd_recall_exact_rows"])
    assert np.all(np.diff(dist, axis=1) >= 0)


def test_c3_fit_trustworthiness_matches_the_reference(c3):
    """The full fit of the benchmark (fit_transform on a host array): trustworthiness@15
    on the fixture's 10,000 rows within 0.005 of the reference embedding's."""
    from mlx_vis_b200 import UMAP
    from mlx_vis_b200.metrics import trustworthiness

    X, g, m = c3
    u = UMAP(n_components=2, n_neighbors=15, min_dist=0.1, n_epochs=500, knn_method="nndescent", random_state=0)
    Y = u.fit_transform(X)
    assert Y.shape == (70000, 2) and np.isfinite(Y).all()
    sub = g["sample"]
    tw = trustworthiness(X[sub], Y[sub], 15)
    assert abs(tw - m["trustworthiness15_sample"]) <= 0.005, (tw, m["trustworthiness15_sample"])
    assert u.graph_info_["n_edges"] == pytest.approx(m["n_edges"], rel=0.01)
