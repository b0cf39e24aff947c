"""Learned warm-start encoder for UMAP: an MLP d -> 512 -> 512 -> c with GELU.

New work (the reference initialises UMAP only spectrally or randomly,
mlx_vis/_umap/umap.py:298-357; its closest idiom is the MMAE MLP trained with
AdamW, mlx_vis/_mmae/mmae.py:22-38, 258-281).  The encoder regresses UMAP
embeddings from the input rows.  Used as ``UMAP(init="learned", encoder=enc)``
it provides the starting layout, so optimize_layout needs fewer epochs, and
``enc.transform(X_new)`` embeds unseen rows without a fit.

Numerics: FP32 master weights and Adam moments; the two hidden layers run as
tcgen05 BF16 GEMMs with FP32 accumulation and fused bias + GELU (erf-based GELU,
erf to 1.5e-7 by Abramowitz & Stegun 7.1.26; libumap_b200 ``umapb_gemm_bf16``);
the c-wide output layer keeps FP32 weights.  The training loss is the mean
squared error per row.  Every step is a sequence of library kernels (forward,
backward with split-K weight gradients, one AdamW launch) — no autograd — and
``fit`` replays it as one CUDA graph per batch.
"""

from __future__ import annotations

import numpy as np
import torch

from mlx_vis_b200 import _lib
from mlx_vis_b200._device import device, to_device_f32, to_host
from mlx_vis_b200._lib import call, ptr, stream_handle

F32, BIAS_GELU, GELU_BACK = 0, 1, 2


def _pad8(x: int) -> int:
    return (x + 7) // 8 * 8


class Encoder:
    """MLP encoder trained on (X, Y) pairs of UMAP embeddings."""

    KSPLIT_MAX = 16

    def __init__(self, in_dim: int, hidden: int = 512, out_dim: int = 2, lr: float = 1e-3,
                 weight_decay: float = 1e-2, betas=(0.9, 0.999), eps: float = 1e-8, batch_size: int = 4096,
                 seed: int = 0):
        if not 1 <= out_dim <= 4:
            raise ValueError("out_dim must be between 1 and 4")
        self.d, self.h, self.c = int(in_dim), int(hidden), int(out_dim)
        self.lr, self.wd, self.betas, self.eps = lr, weight_decay, betas, eps
        self.batch_size = int(batch_size)
        self.seed = seed
        self.step_count = 0
        self.dev = device()
        self.ldx = _pad8(self.d)
        rng = np.random.default_rng(seed)

        def uniform(shape, fan_in):  # the usual Linear initialisation, U(-1/sqrt(fan_in), 1/sqrt(fan_in))
            bound = 1.0 / np.sqrt(fan_in)
            return torch.from_numpy(rng.uniform(-bound, bound, shape).astype(np.float32)).to(self.dev)

        h, d, c = self.h, self.d, self.c
        self.params = {"W1": uniform((h, d), d), "b1": uniform((h,), d), "W2": uniform((h, h), h),
                       "b2": uniform((h,), h), "W3": uniform((c, h), h), "b3": uniform((c,), h)}
        self.m = {k: torch.zeros_like(v) for k, v in self.params.items()}
        self.v = {k: torch.zeros_like(v) for k, v in self.params.items()}
        self.grads = {k: torch.empty_like(v) for k, v in self.params.items()}
        # W1 and W2 gradients arrive as K slices of the split-K GEMMs (AdamW sums them
        # into slice 0, which is grads[...] afterwards)
        self._gpart = {"W1": torch.empty((self.KSPLIT_MAX, h, d), device=self.dev),
                       "W2": torch.empty((self.KSPLIT_MAX, h, h), device=self.dev)}
        for k, t in self._gpart.items():
            self.grads[k] = t[0]
        bf = torch.bfloat16
        self.W1b = torch.zeros((h, self.ldx), dtype=bf, device=self.dev)
        self.W2b = torch.empty((h, h), dtype=bf, device=self.dev)
        self.W2bT = torch.empty((h, h), dtype=bf, device=self.dev)
        self._refresh_bf16()
        self.status = torch.zeros(1, dtype=torch.int32, device=self.dev)
        self.step_t = torch.zeros(1, dtype=torch.int32, device=self.dev)  # AdamW step number on the device
        self._buf = {}
        self.history_ = []
        self.y_scale_ = None  # (mean, std) of the targets the encoder was trained on

    # ------------------------------------------------------------------
    def _refresh_bf16(self):
        p = self.params
        self.W1b[:, : self.d].copy_(p["W1"].to(torch.bfloat16))
        self.W2b.copy_(p["W2"].to(torch.bfloat16))
        self.W2bT.copy_(p["W2"].t().to(torch.bfloat16))

    def _buffers(self, B: int, train: bool):
        key = (B, train)
        if key in self._buf:
            return self._buf[key]
        dev, bf, h, c = self.dev, torch.bfloat16, self.h, self.c
        ldb = _pad8(B)
        b = {"Xb": torch.empty((B, self.ldx), dtype=bf, device=dev), "Z1": torch.empty((B, h), device=dev),
             "H1": torch.empty((B, h), dtype=bf, device=dev), "Z2": torch.empty((B, h), device=dev),
             "H2": torch.empty((B, h), dtype=bf, device=dev), "Y": torch.empty((B, c), device=dev), "ldb": ldb}
        if train:
            b.update({"XT": torch.zeros((self.d, ldb), dtype=bf, device=dev),
                      "H1T": torch.zeros((h, ldb), dtype=bf, device=dev),
                      "dY": torch.empty((B, c), device=dev), "dZ2": torch.empty((B, h), dtype=bf, device=dev),
                      "dZ2T": torch.zeros((h, ldb), dtype=bf, device=dev),
                      "dZ1": torch.empty((B, h), dtype=bf, device=dev),
                      "dZ1T": torch.zeros((h, ldb), dtype=bf, device=dev),
                      "loss": torch.zeros(1, device=dev)})
        self._buf[key] = b
        return b

    def _gemm(self, A, Bm, M, N, K, lda, ldb, epi, C=None, ldc=0, bias=None, Z=None, ldz=0, H=None, ldh=0, HT=None,
              ldt=0, ksplit=1, colsum=None):
        call("umapb_gemm_bf16", ptr(A), ptr(Bm), M, N, K, lda, ldb, epi, ksplit, ptr(C), ldc, ptr(bias), ptr(Z), ldz,
             ptr(H), ldh, ptr(HT), ldt, ptr(colsum), ptr(self.status), stream_handle())

    def _forward(self, X: torch.Tensor, b, train: bool, rows=None):
        B = X.shape[0] if rows is None else rows.numel()
        h, p, s = self.h, self.params, stream_handle()
        call("umapb_mlp_convert", ptr(X), ptr(rows), B, self.d, self.ldx, ptr(b["Xb"]),
             ptr(b["XT"] if train else None), b["ldb"], s)
        self._gemm(b["Xb"], self.W1b, B, h, self.d, self.ldx, self.ldx, BIAS_GELU, bias=p["b1"], Z=b["Z1"], ldz=h,
                   H=b["H1"], ldh=h, HT=b["H1T"] if train else None, ldt=b["ldb"])
        self._gemm(b["H1"], self.W2b, B, h, h, h, h, BIAS_GELU, bias=p["b2"], Z=b["Z2"], ldz=h, H=b["H2"], ldh=h)
        call("umapb_mlp_head_forward", ptr(b["H2"]), h, B, h, ptr(p["W3"]), ptr(p["b3"]), self.c, ptr(b["Y"]), s)
        return b["Y"]

    # ------------------------------------------------------------------
    def train_step(self, X: torch.Tensor, T: torch.Tensor, rows=None) -> torch.Tensor:
        """One AdamW step on a batch; returns the loss (device).  X (B, d) and T (B, c)
        are device float32; with ``rows`` (device int64) they are whole sets and the
        batch is their rows ``rows``, gathered by the kernels."""
        X = X.contiguous()
        T = T.contiguous()
        B = X.shape[0] if rows is None else rows.numel()
        h, d, c, p, g = self.h, self.d, self.c, self.params, self.grads
        b = self._buffers(B, True)
        s = stream_handle()
        ks = self._ksplit(B)
        self._forward(X, b, True, rows)
        # dY, loss, dW3, db3, dZ2 (+ transpose), db2
        call("umapb_mlp_head_backward", ptr(b["Y"]), ptr(T), ptr(rows), B, c, ptr(p["W3"]), h, ptr(b["Z2"]), h,
             ptr(b["H2"]), h, ptr(b["dY"]), ptr(g["W3"]), ptr(g["b3"]), ptr(b["dZ2"]), h, ptr(b["dZ2T"]), b["ldb"],
             ptr(g["b2"]), ptr(b["loss"]), s)
        # dW2 = dZ2^T H1 (K = B in ks slices)
        self._gemm(b["dZ2T"], b["H1T"], h, h, B, b["ldb"], b["ldb"], F32, C=self._gpart["W2"], ldc=h, ksplit=ks)
        # dZ1 = (dZ2 W2) * gelu'(Z1) (+ transpose), db1 = its column sums
        self._gemm(b["dZ2"], self.W2bT, B, h, h, h, h, GELU_BACK, Z=b["Z1"], ldz=h, H=b["dZ1"], ldh=h, HT=b["dZ1T"],
                   ldt=b["ldb"], colsum=g["b1"])
        # dW1 = dZ1^T X (K = B in ks slices)
        self._gemm(b["dZ1T"], b["XT"], h, d, B, b["ldb"], b["ldb"], F32, C=self._gpart["W1"], ldc=d, ksplit=ks)
        self.step_count += 1
        self.step_t.add_(1)
        self._adamw(ks)
        return b["loss"]

    @classmethod
    def _ksplit(cls, K: int) -> int:
        """K slices for the weight-gradient GEMMs (K = batch): about 8 K blocks of 64 each."""
        return max(1, min(cls.KSPLIT_MAX, (K + 511) // 512))

    def _adamw(self, ks: int):
        """One launch for all parameter groups (umapb_adamw); W1 and W2 gradients in ks slices."""
        if getattr(self, "_adamw_args", None) is None:
            import ctypes

            names = list(self.params)
            n = len(names)
            P = ctypes.c_void_p * n
            I = ctypes.c_int32 * n
            bf = {"W1": (self.W1b, self.ldx, None, 0), "W2": (self.W2b, self.h, self.W2bT, self.h)}
            shp = [(t.shape[0], t.shape[1]) if t.dim() == 2 else (1, t.shape[0]) for t in self.params.values()]
            self._adamw_names = names
            self._adamw_stride = (ctypes.c_int64 * n)(*[self.params[k].numel() if k in self._gpart else 0
                                                        for k in names])
            self._adamw_args = (
                n, P(*[ptr(self.params[k]) for k in names]), P(*[ptr(self.grads[k]) for k in names]),
                P(*[ptr(self.m[k]) for k in names]), P(*[ptr(self.v[k]) for k in names]),
                I(*[r for r, _ in shp]), I(*[c for _, c in shp]),
                P(*[ptr(bf[k][0]) if k in bf else None for k in names]), I(*[bf[k][1] if k in bf else 0 for k in names]),
                P(*[ptr(bf[k][2]) if k in bf else None for k in names]), I(*[bf[k][3] if k in bf else 0 for k in names]))
        import ctypes

        slices = (ctypes.c_int32 * len(self._adamw_names))(*[ks if k in self._gpart else 1
                                                             for k in self._adamw_names])
        n, pp, gg, mm, vv, *rest = self._adamw_args
        b1, b2 = self.betas
        call("umapb_adamw", n, pp, gg, slices, self._adamw_stride, mm, vv, *rest, float(self.lr), float(b1), float(b2),
             float(self.eps), float(self.wd), ptr(self.step_t), stream_handle())

    def check_status(self):
        if int(self.status.item()) != 0:
            raise _lib.UmapB200Error("umapb_gemm_bf16", 5, "device-side wait expired in a GEMM")

    # ------------------------------------------------------------------
    def fit(self, Xs, Ys, epochs: int = 20, verbose: bool = False, seed: int = 0, use_graph: bool = True):
        """Trains on the (X, Y) pairs (lists of arrays or tensors); targets are standardised
        with their global mean / std, which transform() undoes.  With ``use_graph`` the
        training step (row gather, forward, backward, AdamW) is recorded once into a
        CUDA graph and replayed for every batch after the first."""
        Xd = torch.cat([to_device_f32(x, self.dev) for x in Xs])
        Yd = torch.cat([to_device_f32(y, self.dev) for y in Ys])
        mean = Yd.mean(dim=0)
        std = Yd.std(dim=0).clamp_min(1e-6)
        self.y_scale_ = (mean, std)
        Yn = ((Yd - mean) / std).contiguous()
        n = Xd.shape[0]
        gen = torch.Generator(device=self.dev)
        gen.manual_seed(seed)
        B = min(self.batch_size, n)
        nb = n // B
        sel = torch.empty(B, dtype=torch.int64, device=self.dev)  # the batch's row indices
        total = torch.zeros((), device=self.dev)

        def step():
            loss = self.train_step(Xd, Yn, rows=sel)
            total.add_(loss[0])

        graph = None
        for ep in range(epochs):
            perm = torch.randperm(n, device=self.dev, generator=gen)
            total.zero_()
            for i in range(nb):
                sel.copy_(perm[i * B:(i + 1) * B])
                if graph is not None:
                    graph.replay()
                    self.step_count += 1
                    continue
                step()  # eager: the first batch (it also sets up every buffer the capture reuses)
                if use_graph and nb * epochs > 1:
                    graph = torch.cuda.CUDAGraph()
                    side = torch.cuda.Stream()
                    side.wait_stream(torch.cuda.current_stream())
                    with torch.cuda.stream(side):
                        count = self.step_count
                        graph.capture_begin()
                        step()
                        graph.capture_end()
                        self.step_count = count  # capturing records the step without running it
                    torch.cuda.current_stream().wait_stream(side)
            self.history_.append(float(total.item()) / max(nb, 1))
            if verbose:
                print(f"encoder epoch {ep + 1}/{epochs}: loss {self.history_[-1]:.4f}")
        self.check_status()
        return self

    def transform_device(self, X: torch.Tensor, chunk: int = 16384) -> torch.Tensor:
        """Embeds rows on the device: (n, c) float32 CUDA tensor in the targets' scale."""
        X = X.contiguous().float()
        out = torch.empty((X.shape[0], self.c), device=self.dev)
        for s0 in range(0, X.shape[0], chunk):
            xb = X[s0:s0 + chunk]
            b = self._buffers(xb.shape[0], False)
            out[s0:s0 + xb.shape[0]].copy_(self._forward(xb, b, False))
        if self.y_scale_ is not None:
            mean, std = self.y_scale_
            out = out * std + mean
        return out

    def transform(self, X) -> np.ndarray:
        """Out-of-sample embedding of new rows (host float32)."""
        return to_host(self.transform_device(to_device_f32(X, self.dev)))

    def init_layout(self, Xd: torch.Tensor) -> torch.Tensor:
        """Starting layout for UMAP(init="learned")."""
        return self.transform_device(Xd).contiguous()

    # ------------------------------------------------------------------
    @classmethod
    def train_on_umap_runs(cls, Xs, n_epochs: int = 200, encoder_epochs: int = 30, finetune_epochs: int = 5,
                           seed: int = 0, umap_kwargs=None, **kw) -> "Encoder":
        """Trains an encoder on UMAP embeddings of the datasets ``Xs`` (same feature space).

        UMAP layouts are defined only up to rotation and reflection, so independent runs
        give targets that disagree with each other.  The runs are therefore chained: the
        first dataset is embedded with the plain (spectral) initialisation, every later
        one with ``init="learned"`` from the encoder trained so far (fine-tuned on each new
        run for ``finetune_epochs``), which keeps all layouts in one orientation.  A fresh
        encoder is then fitted on all pairs for ``encoder_epochs``.
        """
        from mlx_vis_b200._umap.umap import UMAP

        uk = dict(umap_kwargs or {})
        uk.setdefault("knn_method", "nndescent")
        kw.setdefault("out_dim", uk.get("n_components", 2))
        d = int(np.asarray(Xs[0]).shape[1]) if not torch.is_tensor(Xs[0]) else int(Xs[0].shape[1])
        pairs_x, pairs_y = [], []
        enc = None
        for j, X in enumerate(Xs):
            if enc is None:
                Y = UMAP(n_epochs=n_epochs, random_state=seed + j, **uk).fit_transform(X)
                enc = cls(d, seed=seed, **kw).fit([X], [Y], epochs=encoder_epochs)
            else:
                Y = UMAP(n_epochs=n_epochs, random_state=seed + j, init="learned", encoder=enc, **uk).fit_transform(X)
                enc.fit([X], [Y], epochs=finetune_epochs)
            pairs_x.append(X)
            pairs_y.append(Y)
        final = cls(d, seed=seed, **kw).fit(pairs_x, pairs_y, epochs=encoder_epochs)
        final.train_embeddings_ = pairs_y
        return final

    # ------------------------------------------------------------------
    def state_dict(self) -> dict:
        out = {k: to_host(v) for k, v in self.params.items()}
        out["config"] = np.array([self.d, self.h, self.c])
        if self.y_scale_ is not None:
            out["y_mean"], out["y_std"] = to_host(self.y_scale_[0]), to_host(self.y_scale_[1])
        return out

    def save(self, path: str) -> None:
        np.savez(path, **self.state_dict())

    @classmethod
    def load(cls, path: str, **kw) -> "Encoder":
        z = np.load(path)
        d, h, c = (int(v) for v in z["config"])
        enc = cls(d, hidden=h, out_dim=c, **kw)
        for k in enc.params:
            enc.params[k].copy_(torch.from_numpy(z[k]))
        if "y_mean" in z:
            enc.y_scale_ = (torch.from_numpy(z["y_mean"]).to(enc.dev), torch.from_numpy(z["y_std"]).to(enc.dev))
        enc._refresh_bf16()
        return enc
