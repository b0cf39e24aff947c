"""UMAP on one B200 — drop-in for ``mlx_vis.UMAP`` (mlx_vis/_umap/umap.py:25-449).

Same constructor arguments and defaults (umap.py:46-60) and the same
``fit_transform(X, epoch_callback=None)`` contract (umap.py:75-144): host float32
result of shape (n, n_components), stored in ``embedding_``; ``n_epochs``
defaults to 500 for n <= 10000 and 200 above and is written back to the
estimator (umap.py:123-124); ``epoch_callback(epoch, Y)`` is called with epoch 0
and after every epoch that has active edges (umap.py:420-442).

Pipeline, all on the GPU through libumap_b200:
  kNN (brute tcgen05 / NNDescent) -> fuzzy set (FP64 sigma bisection)
  -> spectral init (CSR SpMV + Cholesky-QR power iteration)
  -> layout epochs (exact float32 schedule, synchronous SGD), two launches per
     epoch, run as one CUDA graph that the library records and updates per fit.
Host work left: the a/b curve fit (float64, microseconds); the NumPy streams the
reference draws from are seeded on the host and drawn on the device.

New keyword arguments (defaults keep the reference behaviour):
  init        "spectral" (reference), "random" (N(0, 1e-4) like the reference's
              fallback), or "learned" (the MLP warm start of ``encoder``)
  encoder     a trained ``mlx_vis_b200.encoder.Encoder`` for init="learned"
  use_graph   run the epoch loop as one CUDA graph (no callback only; default).
              The library records it and keeps one executable graph per device,
              updated in place by later fits; False issues the 2 x n_epochs
              launches one by one.
"""

from __future__ import annotations

import os
import time

import numpy as np
import torch

from mlx_vis_b200 import _lib
from mlx_vis_b200._curve import find_ab_params
from mlx_vis_b200._device import device, to_host, upload_blocks_async
from mlx_vis_b200._normalize import normalize_input


def _random_seed() -> int:
    return int.from_bytes(os.urandom(8), "little")


class UMAP:
    """UMAP dimensionality reduction on an NVIDIA B200.

    Parameters mirror mlx_vis.UMAP: n_components, n_neighbors, min_dist, spread,
    n_epochs, learning_rate, negative_sample_rate, random_state, verbose, pca_dim,
    knn_method ("auto" | "brute" | "nndescent"), normalize.
    """

    def __init__(
        self,
        n_components: int = 2,
        n_neighbors: int = 15,
        min_dist: float = 0.1,
        spread: float = 1.0,
        n_epochs: int | None = None,
        learning_rate: float = 1.0,
        negative_sample_rate: int = 5,
        random_state: int | None = None,
        verbose: bool = False,
        pca_dim: int | None = None,
        knn_method: str = "auto",
        normalize: str | bool = False,
        init: str = "spectral",
        encoder=None,
        use_graph: bool = True,
    ):
        self.n_components = n_components
        self.n_neighbors = n_neighbors
        self.min_dist = min_dist
        self.spread = spread
        self.n_epochs = n_epochs
        self.learning_rate = learning_rate
        self.negative_sample_rate = negative_sample_rate
        self.random_state = random_state
        self.verbose = verbose
        self.pca_dim = pca_dim
        self.knn_method = knn_method
        self.normalize = normalize
        self.init = init
        self.encoder = encoder
        self.use_graph = use_graph
        self.embedding_ = None
        self._spectral_ws = None
        self.timings_ = {}
        self.profile_kernels = False  # CUDA events around NNDescent iteration kernels (bench roofline)

    # ------------------------------------------------------------------
    def fit_transform(self, X, epoch_callback=None) -> np.ndarray:
        """Fit UMAP and return the embedding (host float32, (n, n_components))."""
        self._fit(X, epoch_callback, host_out=True)
        return self.embedding_

    def fit_transform_device(self, X, epoch_callback=None) -> torch.Tensor:
        """Like fit_transform but returns the CUDA tensor (no device-to-host copy)."""
        return self._fit(X, epoch_callback, host_out=False)

    def _fit(self, X, epoch_callback, host_out: bool) -> torch.Tensor:
        if self.n_components < 1 or self.n_components > 32:
            raise ValueError("n_components must be between 1 and 32")
        dev = device()
        ev = _Events(dev)
        if self.normalize:
            Xh = X.detach().cpu().numpy() if isinstance(X, torch.Tensor) else np.asarray(X, dtype=np.float32)
            X = normalize_input(np.asarray(Xh, dtype=np.float32), self.normalize).astype(np.float32)
        # a host X is copied on a side stream in row blocks; the draws below and
        # NNDescent's random start do not read X and run while the copy is in
        # flight, and NNDescent prepares each row block once it has arrived
        Xd, x_ready, x_blocks = upload_blocks_async(X, dev)
        n, dim = Xd.shape
        if n < 2:
            raise ValueError("UMAP needs at least 2 samples")
        seed = self.random_state if self.random_state is not None else _random_seed()
        # the spectral init's draws: while a host X is on its way, or (X already on the
        # device, NNDescent) while NNDescent's first iteration runs, where their host
        # work would otherwise leave the device idle
        from mlx_vis_b200._knn import resolve_method

        draws = None
        defer_draws = (self.init == "spectral" and not x_blocks and self.pca_dim is None
                       and resolve_method(self.knn_method, n) == "nndescent")
        if self.init == "spectral" and not defer_draws:
            draws = self._spectral_draws(n, seed, dev)
        ev.mark("upload")

        if self.pca_dim is not None and dim > self.pca_dim:
            x_ready = self._wait(x_ready, dev)
            x_blocks = None
            Xd = self._pca(Xd)
            ev.mark("pca")

        if self.verbose:
            print("Computing nearest neighbors...")
        from mlx_vis_b200._knn import RERANK_EXTRA
        from mlx_vis_b200._nndescent.nndescent import NNDescent

        k = min(self.n_neighbors, n - 1)
        if resolve_method(self.knn_method, n) == "nndescent":  # _knn.py:35-45
            nn = NNDescent(k=k, verbose=self.verbose,
                           random_state=self.random_state if self.random_state is not None else 42)
            nn.profile_kernels = self.profile_kernels
            hook = None
            if defer_draws:
                def hook():
                    nonlocal draws
                    draws = self._spectral_draws(n, seed, dev)
            knn_idx, knn_dist = nn.build_device(Xd, x_ready=x_ready, x_blocks=x_blocks, while_first_iteration=hook)
            if defer_draws and draws is None:  # a build that ran no iteration
                draws = self._spectral_draws(n, seed, dev)
            x_ready = None
            self.nndescent_ = nn
        else:
            x_ready = self._wait(x_ready, dev)
            knn_idx, knn_dist = _lib.knn_brute(Xd, k, extra=RERANK_EXTRA)
            self.nndescent_ = None
        ev.mark("knn")

        if self.n_epochs is None:
            self.n_epochs = 500 if n <= 10000 else 200
        if self.verbose:
            print("Building fuzzy simplicial set...")
        rows, cols, vals, n_edges = _lib.fuzzy(knn_idx, knn_dist, self.n_epochs, fp64=True)
        ev.mark("fuzzy")

        a, b = find_ab_params(self.spread, self.min_dist)
        self.a_, self.b_ = a, b

        if self.verbose:
            print("Initializing embedding...")
        self._spectral_ws = None
        self.init_used_ = self.init
        Y = self._init_embedding(Xd, rows, cols, vals, n_edges, n, seed, draws)
        ev.mark("init")

        self._optimize(rows, cols, vals, n_edges, Y, a, b, n, seed, epoch_callback)
        ev.mark("layout")
        # the values the host reads after the fit (edge count, spectral status, the
        # embedding for fit_transform) are copied into pinned memory on the stream,
        # so one synchronisation serves them all
        ne_h = torch.empty(1, dtype=torch.int64, pin_memory=True)
        ne_h.copy_(n_edges.reshape(-1)[:1], non_blocking=True)
        st_h = None
        if self._spectral_ws is not None:
            st_h = torch.empty(1, dtype=torch.int32, pin_memory=True)
            st_h.copy_(self._spectral_ws[:4].view(torch.int32), non_blocking=True)
        Y_h = None
        if host_out:
            Y_h = torch.empty(Y.shape, dtype=Y.dtype, pin_memory=True)
            Y_h.copy_(Y, non_blocking=True)
        self.timings_ = ev.finish()  # synchronises the device
        self.graph_info_ = {"n_edges": int(ne_h[0])}
        if Y_h is not None:
            self.embedding_ = Y_h.numpy()
        if st_h is not None and int(st_h[0]) != 0:
            # the power iteration's bounded grid barrier gave up; the device already
            # replaced Y by the random start (umap.py:354-357)
            self.init_used_ = "random"
            if self.verbose:
                print("Spectral init failed (grid barrier timed out), used random initialization")
        self._spectral_ws = None
        return Y

    # ------------------------------------------------------------------
    def _pca(self, Xd: torch.Tensor) -> torch.Tensor:
        """Optional PCA (umap.py:92-113): column means, the covariance
        (X - mean)^T (X - mean) / (n - 1) and the projection (X - mean) @ V on the
        tensor cores (split-precision BF16 products with FP32-level error), the
        eigendecomposition on the host in float64 (the reference also runs eigh on
        the CPU, umap.py:98), V = the last pca_dim eigenvectors in reverse order."""
        n, d = Xd.shape
        mean = _lib.colmean(Xd)
        XT3, kpn = _lib.split3(Xd, mu=mean, transpose=True)  # operand rows = features, K = samples
        # K = n rows, cut into slices of at most 1024 rows summed in FP64
        cov = _lib.gemm_split3(XT3, XT3, kpn, scale=1.0 / max(n - 1, 1))
        del XT3
        evals, evecs = np.linalg.eigh(to_host(cov).astype(np.float64))
        proj = np.ascontiguousarray(evecs[:, -self.pca_dim:][:, ::-1], dtype=np.float32)
        self.pca_eigenvalues_ = evals
        if self.verbose:
            ret = float(evals[-self.pca_dim:].sum() / evals.sum())
            print(f"Variance retained: {ret * 100:.1f}%")
        X3 = _lib.split3(Xd, mu=mean)
        return _lib.matmul(Xd, torch.from_numpy(proj).to(Xd.device), A3=X3)

    @staticmethod
    def _wait(x_ready, dev):
        if x_ready is not None:
            torch.cuda.current_stream(dev).wait_event(x_ready)
        return None

    def _spectral_draws(self, n, seed, dev):
        """The spectral init's random inputs, which depend only on n and the seeds:
        V0 (n, c + 1) and the reference's noise RandomState(random_state or
        42).normal(scale=1e-4, size=(n, c)) as float32 (umap.py:344-346), drawn on
        the device from that stream's state."""
        c = self.n_components
        V0 = _lib.normal((n, c + 1), seed, dev)
        noise_d = _lib.legacy_normal(np.random.RandomState(self.random_state or 42), (n, c), 0.0, 0.0001, dev)
        return V0, noise_d

    def _init_embedding(self, Xd, rows, cols, vals, n_edges, n, seed, draws=None) -> torch.Tensor:
        c = self.n_components
        dev = Xd.device
        if self.init == "learned":
            if self.encoder is None:
                raise ValueError("init='learned' needs an encoder")
            return self.encoder.init_layout(Xd)
        if self.init == "random":
            return _lib.normal((n, c), seed, dev) * 0.01
        if self.init != "spectral":
            raise ValueError(f"unknown init {self.init!r}")
        try:
            V0, noise_d = draws if draws is not None else self._spectral_draws(n, seed, dev)
            # a power iteration whose grid barrier gives up is replaced on the device
            # by the random start below (no host round trip); fit_transform reads the
            # status word once the fit is done
            Y, self._spectral_ws = _lib.spectral(rows, cols, vals, n_edges, n, c, V0, noise_d, n_iter=100,
                                                 fallback_seed=seed, return_workspace=True)
            if self.verbose:
                print("Using spectral initialization")
            return Y
        except _lib.UmapB200Error as e:  # the reference falls back to random init (umap.py:354-357)
            if self.verbose:
                print(f"Spectral init failed ({e}), using random initialization")
            self.init_used_ = "random"
            return _lib.normal((n, c), seed, dev) * 0.01

    def _optimize(self, rows, cols, vals, n_edges, Y, a, b, n, seed, epoch_callback):
        ne = int(self.n_epochs)
        lay = _lib.Layout(rows, cols, vals, n_edges, n, self.n_components, ne)
        layout_seed = (seed * 0x9E3779B97F4A7C15 + 1) & 0xFFFFFFFFFFFFFFFF
        args = (a, b, self.learning_rate, self.negative_sample_rate, layout_seed)
        if epoch_callback is not None:
            epoch_callback(0, to_host(Y))
            for e in range(ne):
                if lay.count_active(e) == 0:
                    continue
                lay.epochs(Y, e, e + 1, *args)
                epoch_callback(e + 1, to_host(Y))
                if self.verbose and (e + 1) % 50 == 0:
                    print(f"Epoch {e + 1}/{ne}")
            return
        # by default the whole epoch loop is one CUDA graph, recorded by the library and
        # kept per device (later fits only update its parameters)
        lay.epochs(Y, 0, ne, *args, graph=self.use_graph and ne > 0)
        if self.verbose:
            print(f"Epoch {ne}/{ne}")


class _Events:
    """Per-stage CUDA-event timings (milliseconds) collected without extra syncs,
    with the host time at which each stage finished issuing its work (host_ keys)."""

    def __init__(self, dev):
        self.dev = dev
        self.t0 = time.perf_counter()
        self.start = torch.cuda.Event(enable_timing=True)
        self.start.record()
        self.marks = []
        self.host = []

    def mark(self, name):
        e = torch.cuda.Event(enable_timing=True)
        e.record()
        self.marks.append((name, e))
        self.host.append((name, time.perf_counter()))

    def finish(self):
        torch.cuda.synchronize(self.dev)
        out = {}
        prev = self.start
        for name, e in self.marks:
            out[name] = prev.elapsed_time(e)
            prev = e
        out["total_device"] = self.start.elapsed_time(prev)
        out["total_wall"] = (time.perf_counter() - self.t0) * 1000.0
        t = self.t0
        for name, h in self.host:
            out["host_" + name] = (h - t) * 1000.0
            t = h
        return out
