"""End-to-end UMAP on the GPU through the public API (drop-in for mlx_vis.UMAP)."""

import numpy as np
import pytest
from sklearn.manifold import trustworthiness

pytestmark = pytest.mark.gpu


def test_fit_transform_trustworthiness_matches_reference(gauss2000, manifest):
    from mlx_vis_b200 import UMAP

    ref_tw = manifest["umap_gauss"]["trustworthiness15"]
    u = UMAP(n_components=2, n_neighbors=15, min_dist=0.1, n_epochs=200, knn_method="brute", random_state=0)
    Y = u.fit_transform(gauss2000)
    assert Y.shape == (2000, 2) and Y.dtype == np.float32 and np.isfinite(Y).all()
    assert u.embedding_ is Y
    tw = trustworthiness(gauss2000, Y, n_neighbors=15)
    assert abs(tw - ref_tw) <= 0.005, (tw, ref_tw)
    assert set(u.timings_) >= {"knn", "fuzzy", "init", "layout"}


def test_graph_and_eager_epoch_loops_agree(gauss2000):
    from mlx_vis_b200 import UMAP

    ys = []
    for use_graph in (True, False):
        u = UMAP(n_epochs=50, knn_method="brute", random_state=3, use_graph=use_graph)
        ys.append(u.fit_transform(gauss2000))
    # float atomics reorder sums; the two runs may differ only by rounding-level noise
    tw = [trustworthiness(gauss2000, y, n_neighbors=15) for y in ys]
    assert abs(tw[0] - tw[1]) < 0.003


def test_epoch_callback_semantics(gauss2000, golden):
    from mlx_vis_b200 import UMAP

    seen = []
    u = UMAP(n_epochs=30, knn_method="brute", random_state=0)
    u.fit_transform(gauss2000[:500], epoch_callback=lambda e, Y: seen.append((e, Y.shape, Y.dtype)))
    epochs = [e for e, _, _ in seen]
    assert epochs[0] == 0 and epochs == sorted(epochs) and all(s == (500, 2) for _, s, _ in seen)
    assert 1 not in epochs  # epoch 0 never has active edges, so the first callback after it is epoch 2


def test_n_epochs_default_is_written_back():
    from mlx_vis_b200 import UMAP
    from mlx_vis_b200.datasets import gaussian_mixture

    X = gaussian_mixture(300, 8, seed=1)
    u = UMAP(knn_method="brute", random_state=0)
    u.fit_transform(X)
    assert u.n_epochs == 500


@pytest.mark.parametrize("n_components", [1, 3, 5, 8, 32])
def test_other_output_dims(n_components):
    from mlx_vis_b200 import UMAP
    from mlx_vis_b200.datasets import gaussian_mixture

    X = gaussian_mixture(600, 16, seed=2)
    Y = UMAP(n_components=n_components, n_epochs=60, knn_method="brute", random_state=0).fit_transform(X)
    assert Y.shape == (600, n_components) and np.isfinite(Y).all()


@pytest.mark.parametrize("method", ["nndescent", "brute"])
def test_host_and_device_inputs_give_the_same_fit(gauss2000, method):
    """A host X (NumPy or pinned torch) is uploaded on a side stream while the
    random start and the spectral draws run; the fit matches one from an X already
    on the device up to the layout's float-atomic rounding."""
    import torch

    from mlx_vis_b200 import UMAP

    tw = []
    for X in (gauss2000, torch.from_numpy(gauss2000).cuda(), torch.from_numpy(gauss2000).pin_memory()):
        Y = UMAP(n_epochs=50, knn_method=method, random_state=5).fit_transform(X)
        assert Y.shape == (2000, 2) and np.isfinite(Y).all()
        tw.append(trustworthiness(gauss2000, Y, n_neighbors=15))
    assert max(tw) - min(tw) < 0.003, tw


def test_nndescent_waits_for_the_upload_after_its_random_start(gauss2000):
    import torch

    from mlx_vis_b200 import NNDescent
    from mlx_vis_b200._device import upload_async

    Xd, ready = upload_async(gauss2000)
    assert ready is not None
    idx_a, dist_a = NNDescent(k=15, random_state=7).build_device(Xd, x_ready=ready)
    idx_b, dist_b = NNDescent(k=15, random_state=7).build_device(torch.from_numpy(gauss2000).cuda())
    assert torch.equal(idx_a, idx_b) and torch.equal(dist_a, dist_b)


@pytest.mark.parametrize("d", [64, 350])
def test_nndescent_prepares_row_blocks_as_they_arrive(d):
    """An upload in row blocks (upload_blocks_async): norms, split, both projections
    and FP16 rows are made block by block as the rows arrive; the graph equals the
    one built from a device-resident X (350 features run both projections)."""
    import torch

    from mlx_vis_b200 import NNDescent
    from mlx_vis_b200._device import upload_blocks_async

    X = np.random.default_rng(d).normal(size=(3001, d)).astype(np.float32)
    Xd, done, blocks = upload_blocks_async(torch.from_numpy(X).pin_memory(), blocks=5)
    assert done is not None and len(blocks) == 5 and blocks[-1][0] == 3001
    idx_a, dist_a = NNDescent(k=15, random_state=3).build_device(Xd, x_blocks=blocks)
    idx_b, dist_b = NNDescent(k=15, random_state=3).build_device(torch.from_numpy(X).cuda())
    assert torch.equal(idx_a, idx_b) and torch.equal(dist_a, dist_b)


def test_wide_embedding_keeps_neighbourhoods(gauss2000):
    """n_components above 4 (warp-per-row spectral init, warp-per-edge epochs): the
    embedding of the 10-cluster mixture stays trustworthy like the 2-d one."""
    from mlx_vis_b200 import UMAP

    Y = UMAP(n_components=8, n_epochs=200, knn_method="brute", random_state=0).fit_transform(gauss2000)
    assert Y.shape == (2000, 8) and np.isfinite(Y).all()
    assert trustworthiness(gauss2000, Y, n_neighbors=15) > 0.95


def test_n_components_outside_the_envelope_is_rejected():
    from mlx_vis_b200 import UMAP

    with pytest.raises(ValueError, match="n_components"):
        UMAP(n_components=33).fit_transform(np.zeros((10, 3), dtype=np.float32))


def test_spectral_failure_falls_back_to_the_random_start(gauss2000):
    """The reference falls back to a random start when its spectral init fails
    (umap.py:354-357).  Here the failure is the power iteration's bounded grid
    barrier giving up: a 1 ns limit makes every wait expire (no GPU fault, the
    kernel returns), the device swaps in normal((n, c), seed) * 0.01, and the fit
    reports init_used_ == "random"."""
    import torch

    from mlx_vis_b200 import UMAP, _lib

    n = 20000
    X = np.concatenate([gauss2000] * 10)[:n] + np.random.default_rng(0).normal(scale=0.01, size=(n, 64)).astype(
        np.float32)
    Xd = torch.from_numpy(X.astype(np.float32)).cuda()
    idx, dist = _lib.knn_brute(Xd, 15)
    rows, cols, vals, ne = _lib.fuzzy(idx, dist, 200)
    V0 = _lib.normal((n, 3), 1, Xd.device)
    noise = _lib.normal((n, 2), 2, Xd.device) * 1e-4
    ok, ws_ok = _lib.spectral(rows, cols, vals, ne, n, 2, V0, noise, fallback_seed=9, return_workspace=True)
    assert _lib.status_word(ws_ok) == 0
    try:
        _lib.set_wait_limit_ns(1)
        Y, ws = _lib.spectral(rows, cols, vals, ne, n, 2, V0, noise, fallback_seed=9, return_workspace=True)
        assert _lib.status_word(ws) != 0
        want = _lib.normal((n, 2), 9, Xd.device) * 0.01
        assert torch.equal(Y, want)
        assert not torch.equal(ok, want)
        u = UMAP(n_epochs=20, knn_method="brute", random_state=4)
        Yu = u.fit_transform(Xd)
        assert u.init_used_ == "random" and np.isfinite(Yu).all()
    finally:
        _lib.set_wait_limit_ns(0)
    u = UMAP(n_epochs=20, knn_method="brute", random_state=4)
    u.fit_transform(Xd)
    assert u.init_used_ == "spectral"
