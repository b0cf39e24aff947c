"""Host-side logic that needs no GPU: the a/b curve fit, input normalisation,
method dispatch, the estimator's reference-compatible surface."""

import inspect

import numpy as np
import pytest

from mlx_vis_b200._curve import find_ab_params
from mlx_vis_b200._knn import resolve_method
from mlx_vis_b200._normalize import normalize_input


def test_ab_params_bit_exact(golden):
    g = golden("ab_params")
    for (s, m), (a, b) in zip(g["grid"], g["ab"]):
        assert find_ab_params(s, m) == (a, b)


def test_ab_params_diverging_raises_like_reference(golden):
    g = golden("ab_params")
    for s, m in g["diverging"]:
        with pytest.raises(np.linalg.LinAlgError):
            find_ab_params(s, m)


def test_normalize_modes():
    X = np.random.default_rng(0).normal(size=(50, 4)).astype(np.float32) * 3 + 1
    assert normalize_input(X, False) is X and normalize_input(X, None) is X
    z = normalize_input(X, True)
    np.testing.assert_allclose(z.mean(0), 0, atol=1e-5)
    np.testing.assert_allclose(normalize_input(X, "standard"), z)
    mm = normalize_input(X, "minmax")
    assert mm.min() >= 0 and mm.max() <= 1.0
    with pytest.raises(ValueError, match="Unknown normalize method"):
        normalize_input(X, "zca")


def test_method_dispatch_matches_reference():
    assert resolve_method("auto", 20000) == "brute"
    assert resolve_method("auto", 20001) == "nndescent"
    assert resolve_method("nndescent", 10) == "nndescent"
    assert resolve_method("brute", 10**6) == "brute"
    assert resolve_method("anything-else", 50) == "brute"  # the reference falls through to brute


def test_umap_signature_is_drop_in():
    from mlx_vis_b200 import UMAP

    sig = inspect.signature(UMAP.__init__)
    ref = dict(n_components=2, n_neighbors=15, min_dist=0.1, spread=1.0, n_epochs=None, learning_rate=1.0,
               negative_sample_rate=5, random_state=None, verbose=False, pca_dim=None, knn_method="auto",
               normalize=False)
    for name, default in ref.items():
        assert sig.parameters[name].default == default, name
    names = list(sig.parameters)[1:13]
    assert names == list(ref)  # same positional order as umap.py:46-60
    assert list(inspect.signature(UMAP.fit_transform).parameters) == ["self", "X", "epoch_callback"]


def test_nndescent_signature_is_drop_in():
    from mlx_vis_b200 import NNDescent

    sig = inspect.signature(NNDescent.__init__)
    ref = dict(k=15, n_iters=20, max_candidates=None, delta=0.015, random_state=None, verbose=False)
    assert list(sig.parameters)[1:] == list(ref)
    for name, default in ref.items():
        assert sig.parameters[name].default == default


def test_import_paths():
    import mlx_vis_b200
    from mlx_vis_b200.nndescent import NNDescent
    from mlx_vis_b200.umap import UMAP

    assert mlx_vis_b200.UMAP is UMAP and mlx_vis_b200.NNDescent is NNDescent
    from mlx_vis_b200._knn import compute_knn

    assert list(inspect.signature(compute_knn).parameters) == ["X", "k", "method", "verbose", "random_state",
                                                                "return_euclidean"]


def test_fit_without_gpu_fails_loudly(monkeypatch):
    import torch

    from mlx_vis_b200 import UMAP

    monkeypatch.setattr(torch.cuda, "is_available", lambda: False)
    with pytest.raises(RuntimeError, match="CUDA device"):
        UMAP().fit_transform(np.zeros((10, 3), dtype=np.float32))


@pytest.mark.parametrize("n,k,d,seed", [(50, 5, 120, 3), (300, 15, 400, 7), (2, 1, 5, 1), (1000, 15, 101, 0)])
def test_mt19937_restatement_matches_numpy(n, k, d, seed):
    """The oracle's MT19937 / masked-rejection / polar-normal restatement (the
    checker of the device random start) reproduces NumPy's legacy draws and state."""
    from mlx_vis_b200._nndescent.nndescent import random_start, state_words, words_state
    from oracle import mt19937

    np.random.seed(seed)
    st0 = np.random.get_state()
    idx, P, P2, st = mt19937.random_start(st0, n, k, d)
    idx_h, P_h, P2_h = random_start(n, k, d, seed)
    st_h = np.random.get_state()
    assert np.array_equal(idx, idx_h)
    for a, b in ((P, P_h), (P2, P2_h)):
        assert (a is None and b is None) or np.array_equal(a, b)
    assert np.array_equal(st[1], st_h[1]) and st[2:] == st_h[2:]
    # the uint32 state buffer of umapb_nnd_random_start round-trips
    back = words_state(state_words(st_h))
    assert np.array_equal(back[1], st_h[1]) and back[2:] == st_h[2:]


def test_fit_sampler_scales_full_size_samples():
    """oracle.pipeline.FitSampler (the CPU baseline): every stage runs on the full
    input and each estimate is a positive, finite number of seconds."""
    from mlx_vis_b200.datasets import prototype_mixture
    from oracle import nndescent as onnd
    from oracle.pipeline import FitSampler

    X = prototype_mixture(1200, 64, seed=2)
    (idx, _), log = onnd.build(X, k=10, random_state=0, history=True)
    fs = FitSampler(X, idx, [h["changed"] for h in log], n_epochs=50, block=200, epochs_per_step=2)
    r = fs.step()
    assert set(r) == {"knn", "fuzzy", "init", "layout", "fit"}
    assert all(np.isfinite(v) and v > 0 for v in r.values())
    assert abs(r["fit"] - (r["knn"] + r["fuzzy"] + r["init"] + r["layout"])) < 1e-9
    assert fs.updates_total > 0 and "1200 x 64" in fs.describe()
