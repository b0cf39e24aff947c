"""Learned warm-start encoder: the tcgen05 GEMM, the hand-written forward,
backward and AdamW kernels against float64 references, and training."""

import numpy as np
import pytest
import torch

from oracle import mlp as omlp

pytestmark = pytest.mark.gpu


def gemm(A, B, epi=0, bias=None, Z=None, with_t=False, ksplit=1, colsum=False):
    from mlx_vis_b200 import _lib

    M, K = A.shape
    N = B.shape[0]
    st = torch.zeros(1, dtype=torch.int32, device="cuda")
    Cs = torch.full((ksplit, M, N), float("nan"), device="cuda") if epi == 0 else None  # K slices
    H = torch.empty((M, N), dtype=torch.bfloat16, device="cuda") if epi else None
    HT = torch.empty((N, M), dtype=torch.bfloat16, device="cuda") if (epi and with_t) else None
    Zo = torch.empty((M, N), device="cuda") if epi == 1 else Z
    cs = torch.full((N,), float("nan"), device="cuda") if colsum else None
    _lib.call("umapb_gemm_bf16", _lib.ptr(A), _lib.ptr(B), M, N, K, A.stride(0), B.stride(0), epi, ksplit,
              _lib.ptr(Cs), N, _lib.ptr(bias), _lib.ptr(Zo), N, _lib.ptr(H), N, _lib.ptr(HT), M, _lib.ptr(cs),
              _lib.ptr(st), _lib.stream_handle())
    torch.cuda.synchronize()
    assert int(st.item()) == 0
    C = Cs.sum(0) if Cs is not None else None
    return (C, Zo, H, HT, cs) if colsum else (C, Zo, H, HT)


@pytest.mark.parametrize("ksplit", [1, 8, 48])
@pytest.mark.parametrize("M,N,K", [(300, 200, 104), (4096, 512, 784), (512, 784, 4096), (128, 128, 64), (1, 8, 8),
                                   (512, 512, 4000)])
def test_gemm_f32_matches_float64(M, N, K, ksplit):
    g = torch.Generator().manual_seed(M + N + K)
    A = torch.randn((M, K), generator=g).to(torch.bfloat16)
    B = torch.randn((N, K), generator=g).to(torch.bfloat16)
    C, *_ = gemm(A.cuda(), B.cuda(), ksplit=ksplit)
    ref = A.double() @ B.double().T
    err = (C.cpu().double() - ref).abs().max() / ref.abs().max()
    assert err < 1e-5


def test_gemm_epilogues_match_float64():
    g = torch.Generator().manual_seed(0)
    M, N, K = 777, 300, 200
    A = torch.randn((M, K), generator=g).to(torch.bfloat16)
    B = (torch.randn((N, K), generator=g) * 0.1).to(torch.bfloat16)
    bias = torch.randn(N, generator=g)
    _, Z, H, HT = gemm(A.cuda(), B.cuda(), epi=1, bias=bias.cuda(), with_t=True)
    z = A.double() @ B.double().T + bias.double()
    h = torch.nn.functional.gelu(z)
    assert (Z.cpu().double() - z).abs().max() < 1e-4
    assert (H.cpu().double() - h).abs().max() < 1e-2 * max(1.0, float(h.abs().max()))
    assert torch.equal(HT.cpu(), H.cpu().T)
    # backward epilogue: dZ = C * gelu'(Z), with the column sums of the bf16 values
    _, _, dZ, dZT, cs = gemm(A.cuda(), B.cuda(), epi=2, Z=Z, with_t=True, colsum=True)
    zz = z.clone().requires_grad_(True)
    torch.nn.functional.gelu(zz).backward(torch.ones_like(zz))
    ref = (A.double() @ B.double().T) * zz.grad
    assert (dZ.cpu().double() - ref).abs().max() < 1e-2 * max(1.0, float(ref.abs().max()))
    assert torch.equal(dZT.cpu(), dZ.cpu().T)
    want = dZ.cpu().double().sum(0)
    assert (cs.cpu().double() - want).abs().max() < 1e-4 * max(1.0, float(want.abs().max()))


def _params(enc):
    return {k: v.detach().cpu().numpy().copy() for k, v in enc.params.items()}


@pytest.mark.parametrize("d,B", [(784, 512), (64, 1000)])
def test_train_step_gradients_match_float64_autograd(d, B):
    from mlx_vis_b200.encoder import Encoder

    rng = np.random.default_rng(d)
    X = rng.random((B, d)).astype(np.float32)
    T = rng.normal(size=(B, 2)).astype(np.float32)
    enc = Encoder(d, lr=0.0, weight_decay=0.0, seed=1)
    p0 = _params(enc)
    loss = enc.train_step(torch.from_numpy(X).cuda(), torch.from_numpy(T).cuda())
    enc.check_status()
    ref_loss, ref_g, _ = omlp.loss_and_grads(p0, X, T, bf16_like_gpu=True)
    assert abs(float(loss.item()) - ref_loss) <= 1e-3 * abs(ref_loss)
    for k, gr in ref_g.items():
        got = enc.grads[k].cpu().numpy()
        rel = np.linalg.norm(got - gr) / max(np.linalg.norm(gr), 1e-12)
        assert rel < 2e-2, (k, rel)
    # and close to the exact float64 gradients (BF16 storage is the only gap)
    _, exact_g, _ = omlp.loss_and_grads(p0, X, T, bf16_like_gpu=False)
    for k, gr in exact_g.items():
        rel = np.linalg.norm(enc.grads[k].cpu().numpy() - gr) / max(np.linalg.norm(gr), 1e-12)
        assert rel < 5e-2, (k, rel)


def test_adamw_matches_torch_adamw():
    from mlx_vis_b200.encoder import Encoder

    rng = np.random.default_rng(3)
    X = torch.from_numpy(rng.random((256, 40)).astype(np.float32)).cuda()
    T = torch.from_numpy(rng.normal(size=(256, 2)).astype(np.float32)).cuda()
    enc = Encoder(40, lr=1e-3, weight_decay=1e-2, seed=2)
    p0 = _params(enc)
    enc.train_step(X, T)
    grads = {k: v.cpu().numpy().copy() for k, v in enc.grads.items()}
    want = omlp.adamw_step(p0, grads, lr=1e-3, weight_decay=1e-2)
    for k, w in want.items():
        got = enc.params[k].cpu().numpy()
        assert np.allclose(got, w, rtol=1e-5, atol=1e-7), k
    # the BF16 copies the GEMMs read follow the masters
    assert torch.equal(enc.W2bT.cpu(), enc.W2b.cpu().T)
    assert torch.equal(enc.W1b[:, :40].cpu(), enc.params["W1"].to(torch.bfloat16).cpu())


def test_encoder_fits_a_smooth_map():
    from mlx_vis_b200.encoder import Encoder

    rng = np.random.default_rng(0)
    X = rng.normal(size=(8192, 32)).astype(np.float32)
    Y = np.stack([np.tanh(X[:, 0] + 0.5 * X[:, 1]), np.sin(X[:, 2]) * X[:, 3]], axis=1).astype(np.float32)
    enc = Encoder(32, batch_size=1024, seed=0).fit([X], [Y], epochs=30)
    assert enc.history_[-1] < 0.2 * enc.history_[0]
    pred = enc.transform(X)
    assert np.corrcoef(pred[:, 0], Y[:, 0])[0, 1] > 0.9


def test_gpu_trustworthiness_equals_sklearn():
    from sklearn.manifold import trustworthiness as sk_tw

    from mlx_vis_b200.metrics import trustworthiness

    rng = np.random.default_rng(0)
    X = rng.normal(size=(700, 20))
    Y = X[:, :2] + 0.3 * rng.normal(size=(700, 2))
    assert abs(trustworthiness(X, Y, 15) - sk_tw(X, Y, n_neighbors=15)) < 1e-9


def test_learned_init_matches_full_run_trust_in_40pct_of_epochs():
    """Warm start from an encoder trained on other draws of the same distribution:
    200 layout epochs (40%) reach the trustworthiness of a 500-epoch spectral run."""
    from mlx_vis_b200 import UMAP
    from mlx_vis_b200.datasets import prototype_mixture
    from mlx_vis_b200.encoder import Encoder
    from mlx_vis_b200.metrics import trustworthiness

    Xs = [prototype_mixture(5000, 784, seed=j, proto_seed=0) for j in range(1, 5)]
    enc = Encoder.train_on_umap_runs(Xs, n_epochs=200, encoder_epochs=30, umap_kwargs={"knn_method": "brute"})
    Xt = prototype_mixture(10000, 784, seed=100, proto_seed=0)
    sub = np.random.default_rng(0).choice(10000, 4000, replace=False)
    full = UMAP(n_epochs=500, random_state=0).fit_transform(Xt)
    warm = UMAP(n_epochs=200, random_state=0, init="learned", encoder=enc).fit_transform(Xt)
    t_full = trustworthiness(Xt[sub], full[sub], 15)
    t_warm = trustworthiness(Xt[sub], warm[sub], 15)
    assert t_warm >= t_full - 0.005, (t_warm, t_full)
