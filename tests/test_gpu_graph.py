"""Fuzzy simplicial set, spectral initialisation and layout epochs on the GPU
against the reference's golden vectors and the CPU oracle."""

import numpy as np
import pytest
import torch

from oracle import fuzzy as ofz
from oracle import layout as olay
from oracle import spectral as ospec

pytestmark = pytest.mark.gpu


def cuda(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def gpu_fuzzy(idx, dist, n_epochs, fp64):
    from mlx_vis_b200 import _lib

    r, c, v, ne, rho, sig = _lib.fuzzy(cuda(idx.astype(np.int32)), cuda(dist.astype(np.float32)), n_epochs,
                                       fp64=fp64, with_sigma=True)
    E = int(ne.item())
    return (r[:E].cpu().numpy(), c[:E].cpu().numpy(), v[:E].cpu().numpy()), (rho.cpu().numpy(), sig.cpu().numpy())


@pytest.mark.parametrize("name,n_epochs", [("fuzzy_gauss", 200), ("fuzzy_dups", 500)])
def test_fuzzy_fp64_matches_fp64_oracle(name, n_epochs, golden):
    g = golden(name)
    if name == "fuzzy_gauss":
        kb = golden("knn_brute_gauss")
        idx, dist = kb["idx"], kb["dist"]
    else:
        idx, dist = g["knn_idx"], g["knn_dist"]
    (r, c, v), (rho, sig) = gpu_fuzzy(idx, dist, n_epochs, fp64=True)
    (ro, co, vo), (rho_o, sig_o) = ofz.fuzzy_simplicial_set(idx, dist, n_epochs, dtype=np.float64)
    assert np.array_equal(r, ro) and np.array_equal(c, co)
    np.testing.assert_allclose(v, vo, rtol=1e-6)
    np.testing.assert_allclose(sig, sig_o.astype(np.float32), rtol=1e-6)
    # and against the reference (float32 bisection): same edge set, weights within its tolerance band
    assert np.array_equal(r, g["rows"]) and np.array_equal(c, g["cols"])
    rel = np.abs(v - g["vals"]) / g["vals"]
    assert rel.max() < 5e-5 and np.mean(rel < 1e-5) > 0.99


@pytest.mark.parametrize("name,n_epochs", [("fuzzy_gauss", 200), ("fuzzy_dups", 500)])
def test_fuzzy_fp32_mode_matches_reference(name, n_epochs, golden):
    g = golden(name)
    if name == "fuzzy_gauss":
        kb = golden("knn_brute_gauss")
        idx, dist = kb["idx"], kb["dist"]
    else:
        idx, dist = g["knn_idx"], g["knn_dist"]
    (r, c, v), _ = gpu_fuzzy(idx, dist, n_epochs, fp64=False)
    assert np.array_equal(r, g["rows"]) and np.array_equal(c, g["cols"])
    rel = np.abs(v - g["vals"]) / g["vals"]
    # expf and the row-sum order differ from NumPy's by ulps, which can move the
    # stopping point of a few rows inside the 1e-5 convergence band
    assert np.mean(rel <= 1e-5) > 0.99 and rel.max() < 5e-5


@pytest.fixture(params=["coop", "launches"])
def spectral_path(request, monkeypatch):
    """The power iteration runs as one cooperative launch unless UMAPB_SPECTRAL_COOP=0
    selects one launch per iteration; both must agree with the reference."""
    monkeypatch.setenv("UMAPB_SPECTRAL_COOP", "1" if request.param == "coop" else "0")
    return request.param


def test_spectral_matches_reference_with_injected_draws(golden, spectral_path):
    from mlx_vis_b200 import _lib

    fz, sp = golden("fuzzy_gauss"), golden("spectral_gauss")
    n = 2000
    rows, cols, vals = cuda(fz["rows"]), cuda(fz["cols"]), cuda(fz["vals"])
    ne = torch.tensor([rows.numel()], dtype=torch.int64, device="cuda")
    noise = np.random.RandomState(42).normal(scale=0.0001, size=(n, 2)).astype(np.float32)
    Y = _lib.spectral(rows, cols, vals, ne, n, 2, cuda(sp["V0"]), cuda(noise), n_iter=100,
                      check=True).cpu().numpy()
    Y64 = ospec.spectral_init(fz["rows"], fz["cols"], fz["vals"], n, sp["V0"], 0, dtype=np.float64)
    assert np.abs(Y - Y64).max() < 1e-4
    assert np.abs(Y - sp["Y0"]).max() < 1e-3


@pytest.mark.parametrize("dim", [1, 2, 3, 4])
def test_spectral_paths_agree_for_every_dim(golden, monkeypatch, dim):
    """Cooperative and per-iteration power iterations: same sums in FP64, the same
    embedding up to the order of the Gram matrix's atomic additions."""
    from mlx_vis_b200 import _lib

    fz = golden("fuzzy_gauss")
    n = 2000
    rows, cols, vals = cuda(fz["rows"]), cuda(fz["cols"]), cuda(fz["vals"])
    ne = torch.tensor([rows.numel()], dtype=torch.int64, device="cuda")
    V0 = np.random.RandomState(dim).normal(size=(n, dim + 1)).astype(np.float32)
    noise = np.random.RandomState(42).normal(scale=0.0001, size=(n, dim)).astype(np.float32)
    out = {}
    for path in ("1", "0"):
        monkeypatch.setenv("UMAPB_SPECTRAL_COOP", path)
        out[path] = _lib.spectral(rows, cols, vals, ne, n, dim, cuda(V0), cuda(noise), n_iter=100,
                                  check=True).cpu().numpy()
    assert out["1"].shape == (n, dim) and np.all(np.isfinite(out["1"]))
    assert np.abs(out["1"] - out["0"]).max() < 1e-3


@pytest.mark.parametrize("dim", [5, 8, 32])
def test_wide_spectral_matches_fp64_oracle(golden, dim):
    """n_components above 4: one launch per power iteration, one warp per row, the
    Gram matrix factored by the last block; against the FP64 oracle of umap.py:298-348."""
    from mlx_vis_b200 import _lib

    fz = golden("fuzzy_gauss")
    n = 2000
    rows, cols, vals = cuda(fz["rows"]), cuda(fz["cols"]), cuda(fz["vals"])
    ne = torch.tensor([rows.numel()], dtype=torch.int64, device="cuda")
    V0 = np.random.RandomState(dim).normal(size=(n, dim + 1)).astype(np.float32)
    noise = np.random.RandomState(42).normal(scale=0.0001, size=(n, dim)).astype(np.float32)
    Y = _lib.spectral(rows, cols, vals, ne, n, dim, cuda(V0), cuda(noise), n_iter=100, check=True).cpu().numpy()
    V = ospec.power_iteration(fz["rows"], fz["cols"], fz["vals"], n, V0, dtype=np.float64)
    Y64 = ospec.rescale(V[:, 1:].astype(np.float32), 42)
    assert Y.shape == (n, dim)
    # columns whose eigenvalues nearly coincide converge slowly in both; compare the
    # well-separated leading columns tightly and all columns on the whole
    assert np.abs(Y[:, :2] - Y64[:, :2]).max() < 1e-3
    assert np.median(np.abs(Y - Y64)) < 1e-3


def _layout(fz, n=2000, n_epochs=200, dim=2):
    from mlx_vis_b200 import _lib

    rows, cols, vals = cuda(fz["rows"]), cuda(fz["cols"]), cuda(fz["vals"])
    ne = torch.tensor([rows.numel()], dtype=torch.int64, device="cuda")
    return _lib.Layout(rows, cols, vals, ne, n, dim, n_epochs)


def test_schedule_active_counts_match_reference(golden, manifest):
    fz, opt = golden("fuzzy_gauss"), golden("optimize_gauss")
    m = manifest["optimize_gauss"]
    lay = _layout(fz)
    Y = cuda(opt["Y_ep0"].copy())
    counts = []
    for e in range(200):
        counts.append(lay.count_active(e))
        lay.epochs(Y, e, e + 1, m["a"], m["b"], 1.0, 5, 1234)
    assert counts == list(opt["n_active"])


def test_injected_epochs_match_reference(golden, manifest):
    fz, opt = golden("fuzzy_gauss"), golden("optimize_gauss")
    m = manifest["optimize_gauss"]
    lay = _layout(fz)
    Y = cuda(opt["Y_ep0"].copy())
    nonempty = [e for e in range(200) if opt["n_active"][e] > 0]
    assert nonempty[:2] == [1, 2]  # the fixture holds snapshots after epochs 1 and 2 (Y_ep2, Y_ep3)
    scale = float(np.abs(opt["Y_ep0"]).max())
    for j, e in enumerate(nonempty[:2]):
        # epochs before the first non-empty one do nothing
        lay.epochs(Y, (nonempty[j - 1] + 1) if j else 0, e, m["a"], m["b"], 1.0, 5, 0)
        lay.epoch_injected(Y, e, m["a"], m["b"], 1.0, 5, cuda(opt[f"neg_{j}"].astype(np.int32)))
        if j == 0:
            got = Y.cpu().numpy()
            ref = opt[f"Y_ep{e + 1}"]
            # one epoch: within 1e-5 of the reference coordinates (relative to their scale)
            assert np.abs(got - ref).max() <= 1e-5 * max(1.0, scale), np.abs(got - ref).max()
            sets = olay.active_sets(fz["vals"], 200)
            Yo = olay.sgd_epoch(opt["Y_ep0"], fz["rows"][sets[e]], fz["cols"][sets[e]],
                                np.resize(fz["rows"][sets[e]], 5 * len(sets[e])), opt["neg_0"].astype(np.int64),
                                1.0 * (1 - e / 200), m["a"], m["b"])
            assert np.abs(got - Yo).max() <= 1e-5 * max(1.0, scale)
    got = Y.cpu().numpy()
    ref = opt["Y_ep3"]
    # after a second epoch the steep short-range forces amplify rounding; stay close
    assert np.median(np.abs(got - ref)) < 1e-5 and np.abs(got - ref).max() < 1e-2


@pytest.mark.parametrize("dim", [5, 8, 32])
def test_wide_injected_epoch_matches_oracle(golden, manifest, dim):
    """One epoch at n_components above 4 (one warp per edge) with injected tails,
    against the FP32 oracle of umap.py:359-387."""
    fz, opt = golden("fuzzy_gauss"), golden("optimize_gauss")
    m = manifest["optimize_gauss"]
    lay = _layout(fz, dim=dim)
    rng = np.random.default_rng(dim)
    Y0 = rng.uniform(0, 10, size=(2000, dim)).astype(np.float32)
    Y = cuda(Y0.copy())
    sets = olay.active_sets(fz["vals"], 200)
    e = next(t for t in range(200) if len(sets[t]) > 0)
    lay.epochs(Y, 0, e, m["a"], m["b"], 1.0, 5, 0)
    A = len(sets[e])
    neg = rng.integers(0, 2000, 5 * A).astype(np.int32)
    lay.epoch_injected(Y, e, m["a"], m["b"], 1.0, 5, cuda(neg))
    got = Y.cpu().numpy()
    Yo = olay.sgd_epoch(Y0, fz["rows"][sets[e]], fz["cols"][sets[e]], np.resize(fz["rows"][sets[e]], 5 * A),
                        neg.astype(np.int64), 1.0 * (1 - e / 200), m["a"], m["b"])
    assert np.abs(got - Y0).max() > 1e-3  # the epoch moved the points
    assert np.abs(got - Yo).max() <= 1e-4, np.abs(got - Yo).max()


def test_injected_negative_count_is_checked(golden, manifest):
    from mlx_vis_b200 import _lib

    fz, opt = golden("fuzzy_gauss"), golden("optimize_gauss")
    m = manifest["optimize_gauss"]
    lay = _layout(fz)
    Y = cuda(opt["Y_ep0"].copy())
    with pytest.raises(_lib.UmapB200Error, match="negatives are needed"):
        lay.epoch_injected(Y, 1, m["a"], m["b"], 1.0, 5, cuda(opt["neg_0"][:-5].astype(np.int32)))


@pytest.mark.parametrize("parallel", [True, False])
@pytest.mark.parametrize("seed,shape", [(42, (70000, 2)), (0, (1, 3)), (7, (2001, 2)), (3, (1, 1))])
def test_device_legacy_normal_equals_numpy(seed, shape, parallel):
    """The spectral init's noise, RandomState(seed).normal(scale=1e-4) as float32,
    drawn on the device from the stream's state, bit for bit."""
    from mlx_vis_b200 import _lib

    want = np.random.RandomState(seed).normal(scale=0.0001, size=shape).astype(np.float32)
    got = _lib.legacy_normal(np.random.RandomState(seed), shape, 0.0, 0.0001, torch.device("cuda"), parallel=parallel)
    assert np.array_equal(got.cpu().numpy(), want)


def test_graph_epochs_match_launched_epochs(golden, manifest):
    """umapb_layout_epochs_graph (recorded once, then updated in place for a new
    layout) reaches the same coordinates as the launch-by-launch loop; float atomics
    may add the moves of one point in another order, hence the tolerance."""
    fz, opt = golden("fuzzy_gauss"), golden("optimize_gauss")
    m = manifest["optimize_gauss"]
    outs = []
    for graph in (False, True, True):  # the second graph call updates the cached executable
        lay = _layout(fz)
        Y = cuda(opt["Y_ep0"].copy())
        lay.epochs(Y, 0, 6, m["a"], m["b"], 1.0, 5, 7, graph=graph)
        outs.append(Y.cpu().numpy())
    scale = float(np.abs(outs[0]).max())
    assert np.abs(outs[0] - opt["Y_ep0"]).max() > 1e-3 * scale  # the epochs moved the points
    for o in outs[1:]:
        assert np.median(np.abs(o - outs[0])) < 1e-5 * scale
        assert np.abs(o - outs[0]).max() < 1e-2 * scale


@pytest.mark.parametrize("dim", [2, 3])
def test_neg5_kernel_matches_general_kernel(golden, manifest, monkeypatch, dim):
    """At the default 5 negatives per edge the epochs run on a kernel compiled for that
    rate (UMAPB_LAYOUT_NEG5=0 selects the general kernel): both draw the same tails and
    make the same sums, so only the order of the float atomics may differ."""
    fz, opt = golden("fuzzy_gauss"), golden("optimize_gauss")
    m = manifest["optimize_gauss"]
    Y0 = opt["Y_ep0"]
    if dim != Y0.shape[1]:
        Y0 = np.concatenate([Y0, Y0[:, :1] * 0.5], axis=1)[:, :dim].astype(np.float32)
    outs = []
    for flag in ("1", "0"):
        monkeypatch.setenv("UMAPB_LAYOUT_NEG5", flag)
        lay = _layout(fz, dim=dim)
        Y = cuda(Y0.copy())
        lay.epochs(Y, 0, 6, m["a"], m["b"], 1.0, 5, 11, graph=False)
        outs.append(Y.cpu().numpy())
    scale = float(np.abs(outs[0]).max())
    assert np.abs(outs[0] - Y0).max() > 1e-3 * scale
    assert np.median(np.abs(outs[1] - outs[0])) < 1e-5 * scale
    assert np.abs(outs[1] - outs[0]).max() < 1e-2 * scale
