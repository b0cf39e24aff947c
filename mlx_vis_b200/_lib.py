"""ctypes binding of libumap_b200.so (declared in include/umap_b200.h).

PyTorch provides device memory and streams; every compute step is a kernel of
libumap_b200.  There is no fallback: if the library is missing or a call fails,
an exception is raised.
"""

from __future__ import annotations

import ctypes
import os
import threading

import numpy as np
import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libumap_b200.so")

_c = ctypes
_i32, _i64, _u64, _f32, _f64, _sz = _c.c_int32, _c.c_int64, _c.c_uint64, _c.c_float, _c.c_double, _c.c_size_t
_p = _c.c_void_p
_psz = _c.POINTER(_c.c_size_t)

# name -> argtypes (all functions return int status unless listed in _RESTYPES)
SIGNATURES = {
    "umapb_last_error": [],
    "umapb_abi_version": [],
    "umapb_read_status": [_p, _p],
    "umapb_set_wait_limit_ns": [_c.c_ulonglong],
    "umapb_knn_brute_workspace": [_i64, _i64, _i32, _i32, _psz],
    "umapb_knn_brute": [_p, _i64, _i64, _i32, _i32, _i32, _p, _p, _p, _sz, _p],
    "umapb_knn_brute_noalloc": [_p, _i64, _i64, _i32, _i32, _i32, _p, _p, _p, _p],
    "umapb_knn_brute_timed": [_p, _i64, _i64, _i32, _i32, _i32, _p, _p, _p, _sz, _p, _p],
    "umapb_knn_brute_rows_workspace": [_i64, _i64, _i32, _i32, _i64, _i64, _psz],
    "umapb_knn_brute_rows": [_p, _i64, _i64, _i32, _i32, _i32, _i64, _i64, _p, _p, _p, _sz, _p],
    "umapb_fuzzy_workspace": [_i64, _i32, _psz],
    "umapb_fuzzy": [_p, _p, _i64, _i32, _i32, _i32, _p, _p, _p, _p, _p, _p, _p, _sz, _p],
    "umapb_normal_fill": [_p, _i64, _u64, _p],
    "umapb_spectral_workspace": [_i64, _i32, _i64, _i32, _psz],
    "umapb_spectral": [_p, _p, _p, _p, _i64, _i64, _i32, _p, _i32, _p, _p, _p, _sz, _p],
    "umapb_spectral_fallback": [_p, _p, _i64, _i32, _u64, _p],
    "umapb_layout_workspace": [_i64, _i32, _i64, _psz],
    "umapb_layout_prepare": [_p, _p, _i64, _i32, _p, _p, _p, _sz, _p],
    "umapb_layout_epochs": [_p, _i64, _i32, _p, _p, _p, _p, _p, _i64, _i32, _i32, _i32, _f32, _f32, _f32, _i32,
                            _u64, _p, _sz, _p],
    "umapb_layout_epochs_graph": [_p, _i64, _i32, _p, _p, _p, _p, _p, _i64, _i32, _i32, _i32, _f32, _f32, _f32,
                                  _i32, _u64, _p, _sz, _p],
    "umapb_nnd_sqnorms": [_p, _i64, _i32, _i32, _p, _p],
    "umapb_nnd_to_half": [_p, _i64, _i32, _i32, _p, _p],
    "umapb_nnd_gather": [_p, _p, _i64, _i32, _p, _p, _i32, _i32, _p],
    "umapb_nnd_gather_pairs": [_p, _p, _i64, _i32, _p, _p, _i32, _i64, _i64, _p],
    "umapb_nnd_sort_rows": [_p, _p, _i64, _i32, _p],
    "umapb_nnd_reverse_workspace": [_i64, _i32, _psz],
    "umapb_nnd_reverse": [_p, _i64, _i32, _p, _p, _sz, _p],
    "umapb_nnd_join_workspace": [_i64, _i32, _i32, _psz],
    "umapb_nnd_join": [_p, _p, _i32, _i32, _i32, _p, _p, _i64, _i32, _i32, _i32, _p, _p, _p, _p, _p, _sz, _p],
    "umapb_nnd_join_new": [_p, _p, _i32, _p, _p, _p, _i64, _i32, _i32, _i32, _p, _p, _p, _sz, _p],
    "umapb_nnd_iteration": [_p, _p, _i32, _i32, _i32, _p, _p, _p, _p, _p, _p, _p, _i64, _i32, _i32, _i32, _i32, _i32, _p,
                            _p,
                            _p, _p, _p, _p],
    "umapb_kernel_launches": [],
    "umapb_gemm_bf16": [_p, _p, _i32, _i32, _i32, _i32, _i32, _i32, _i32, _p, _i32, _p, _p, _i32, _p, _i32, _p,
                        _i32, _p, _p, _p],
    "umapb_mlp_convert": [_p, _p, _i32, _i32, _i32, _p, _p, _i32, _p],
    "umapb_mlp_head_forward": [_p, _i32, _i32, _i32, _p, _p, _i32, _p, _p],
    "umapb_mlp_head_backward": [_p, _p, _p, _i32, _i32, _p, _i32, _p, _i32, _p, _i32, _p, _p, _p, _p, _i32, _p,
                                _i32, _p, _p, _p],
    "umapb_adamw": [_i32, _p, _p, _p, _p, _p, _p, _p, _p, _p, _p, _p, _p, _f32, _f32, _f32, _f32, _f32, _p, _p],
    "umapb_nnd_sqrt": [_p, _i64, _p, _p],
    "umapb_nnd_random_start_workspace": [_i64, _i32, _i32, _i32, _i32, _psz],
    "umapb_nnd_random_start": [_p, _i64, _i32, _i32, _p, _p, _i32, _p, _i32, _p, _sz, _p],
    "umapb_mt_jump_poly": [_i32, _p, _c.POINTER(_i64)],
    "umapb_probe_random_access": [_p, _p, _i64, _i32, _i64, _i32, _i32, _p, _p],
    "umapb_probe_row_gather": [_p, _i64, _i32, _p, _i64, _p, _p],
    "umapb_legacy_normal_workspace": [_i64, _psz],
    "umapb_legacy_normal": [_p, _i64, _f64, _f64, _p, _p, _sz, _p],
    "umapb_layout_count_active": [_p, _p, _i64, _i32, _i64, _i32, _p, _p, _sz, _p],
    "umapb_split3": [_p, _i64, _i64, _i64, _p, _i32, _i32, _p, _p],
    "umapb_gemm_split3": [_p, _p, _i32, _i32, _i32, _i32, _p, _i32, _p, _p],
    "umapb_colmean_workspace": [_i64, _i64, _psz],
    "umapb_colmean": [_p, _i64, _i64, _i64, _p, _p, _sz, _p],
    "umapb_sum_slices": [_p, _i32, _i64, _f32, _p, _p],
    "umapb_sort_keys_workspace": [_i64, _psz],
    "umapb_sort_keys": [_p, _i64, _i64, _p, _p, _sz, _p],
    "umapb_layout_epoch_injected": [_p, _i64, _i32, _p, _p, _p, _p, _p, _i64, _i32, _i32, _f32, _f32, _f32, _i32,
                                    _p, _i64, _p, _sz, _p],
}
_RESTYPES = {"umapb_last_error": _c.c_char_p, "umapb_kernel_launches": _c.c_ulonglong}


def kernel_launches() -> int:
    """Kernels this library has enqueued in this process (graph captures count once)."""
    return int(load().umapb_kernel_launches())

_lock = threading.Lock()
_lib = None


class UmapB200Error(RuntimeError):
    """A libumap_b200 call returned a non-zero status."""

    def __init__(self, func: str, status: int, message: str):
        super().__init__(f"{func} failed with status {status}: {message}")
        self.func = func
        self.status = status


def load() -> ctypes.CDLL:
    """Loads the library once and declares every signature."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m mlx_vis_b200.build` "
                                   "(the CUDA kernels are required; there is no CPU fallback)")
            lib = ctypes.CDLL(LIB_PATH)
            for name, argtypes in SIGNATURES.items():
                fn = getattr(lib, name)
                fn.argtypes = argtypes
                fn.restype = _RESTYPES.get(name, _c.c_int)
            _lib = lib
    return _lib


def call(name: str, *args) -> None:
    lib = load()
    status = getattr(lib, name)(*args)
    if status != 0:
        msg = lib.umapb_last_error().decode(errors="replace")
        raise UmapB200Error(name, status, msg)


def query(name: str, *args) -> int:
    out = ctypes.c_size_t(0)
    call(name, *args, ctypes.byref(out))
    return int(out.value)


def ptr(t) -> ctypes.c_void_p:
    if t is None:
        return ctypes.c_void_p(0)
    if not t.is_cuda:
        raise ValueError("expected a CUDA tensor")
    if not t.is_contiguous():
        raise ValueError("expected a contiguous tensor")
    return ctypes.c_void_p(t.data_ptr())


def stream_handle(stream=None) -> ctypes.c_void_p:
    s = torch.cuda.current_stream() if stream is None else stream
    return ctypes.c_void_p(s.cuda_stream)


def workspace(nbytes: int, device) -> torch.Tensor:
    return torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=device)


def read_status(ws: torch.Tensor, stream=None) -> None:
    """Synchronises the stream and raises if a kernel reported a device-side failure."""
    call("umapb_read_status", ptr(ws), stream_handle(stream))


# ---------------------------------------------------------------------------
# thin typed wrappers over the C ABI (device tensors in, device tensors out)
# ---------------------------------------------------------------------------

def _require(t: torch.Tensor, dtype, ndim=None, name="tensor"):
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise ValueError(f"{name} must be a CUDA tensor")
    if t.dtype != dtype:
        raise ValueError(f"{name} must be {dtype}, got {t.dtype}")
    if ndim is not None and t.dim() != ndim:
        raise ValueError(f"{name} must have {ndim} dimensions")
    return t.contiguous()


def knn_brute(X: torch.Tensor, k: int, extra: int = 16, squared: bool = False, check: bool = True):
    """Exact kNN of the rows of X (n, d) float32: (idx int32 (n,k), dist float32 (n,k))."""
    X = _require(X, torch.float32, 2, "X")
    n, d = X.shape
    nbytes = query("umapb_knn_brute_workspace", n, d, k, extra)
    ws = workspace(nbytes, X.device)
    idx = torch.empty((n, k), dtype=torch.int32, device=X.device)
    dist = torch.empty((n, k), dtype=torch.float32, device=X.device)
    call("umapb_knn_brute", ptr(X), n, d, k, extra, int(squared), ptr(idx), ptr(dist), ptr(ws), ws.numel(),
         stream_handle())
    if check:
        read_status(ws)
    return idx, dist


def knn_brute_rows(X: torch.Tensor, k: int, row_begin: int, row_count: int, extra: int = 16,
                   squared: bool = False, check: bool = True):
    """kNN of the rows [row_begin, row_begin + row_count) of X against all rows:
    (idx int32 (row_count, k), dist float32 (row_count, k))."""
    X = _require(X, torch.float32, 2, "X")
    n, d = X.shape
    ws = workspace(query("umapb_knn_brute_rows_workspace", n, d, k, extra, row_begin, row_count), X.device)
    idx = torch.empty((row_count, k), dtype=torch.int32, device=X.device)
    dist = torch.empty((row_count, k), dtype=torch.float32, device=X.device)
    call("umapb_knn_brute_rows", ptr(X), n, d, k, extra, int(squared), row_begin, row_count, ptr(idx), ptr(dist),
         ptr(ws), ws.numel(), stream_handle())
    if check:
        read_status(ws)
    return idx, dist


def knn_brute_timed(X: torch.Tensor, k: int, extra: int = 16):
    """knn_brute with CUDA events between its launches: (idx, dist, [prep, tiles,
    rerank] milliseconds); synchronises."""
    X = _require(X, torch.float32, 2, "X")
    n, d = X.shape
    ws = workspace(query("umapb_knn_brute_workspace", n, d, k, extra), X.device)
    idx = torch.empty((n, k), dtype=torch.int32, device=X.device)
    dist = torch.empty((n, k), dtype=torch.float32, device=X.device)
    ms = (_c.c_float * 3)()
    call("umapb_knn_brute_timed", ptr(X), n, d, k, extra, 0, ptr(idx), ptr(dist), ptr(ws), ws.numel(),
         _c.cast(ms, _c.c_void_p), stream_handle())
    read_status(ws)
    return idx, dist, [float(v) for v in ms]


def fuzzy(knn_idx: torch.Tensor, knn_dist: torch.Tensor, n_epochs: int, fp64: bool = True,
          with_sigma: bool = False):
    """Fuzzy simplicial set: (rows, cols, vals, n_edges) with capacity n*k; n_edges is a
    device int64 tensor of shape (1,).  With ``with_sigma`` also returns (rho, sigma)."""
    knn_idx = _require(knn_idx, torch.int32, 2, "knn_idx")
    knn_dist = _require(knn_dist, torch.float32, 2, "knn_dist")
    n, k = knn_idx.shape
    dev = knn_idx.device
    ws = workspace(query("umapb_fuzzy_workspace", n, k), dev)
    rows = torch.empty(n * k, dtype=torch.int32, device=dev)
    cols = torch.empty(n * k, dtype=torch.int32, device=dev)
    vals = torch.empty(n * k, dtype=torch.float32, device=dev)
    n_edges = torch.zeros(1, dtype=torch.int64, device=dev)
    rho = torch.empty(n, dtype=torch.float32, device=dev) if with_sigma else None
    sigma = torch.empty(n, dtype=torch.float32, device=dev) if with_sigma else None
    call("umapb_fuzzy", ptr(knn_idx), ptr(knn_dist), n, k, int(n_epochs), int(bool(fp64)), ptr(rows), ptr(cols),
         ptr(vals), ptr(n_edges), ptr(rho), ptr(sigma), ptr(ws), ws.numel(), stream_handle())
    if with_sigma:
        return rows, cols, vals, n_edges, rho, sigma
    return rows, cols, vals, n_edges


def normal(shape, seed: int, device) -> torch.Tensor:
    """Standard normal float32 tensor drawn by the library's Philox kernel."""
    out = torch.empty(shape, dtype=torch.float32, device=device)
    call("umapb_normal_fill", ptr(out), out.numel(), int(seed) & 0xFFFFFFFFFFFFFFFF, stream_handle())
    return out


def legacy_normal(rs, shape, loc: float, scale: float, device, parallel: bool = True) -> torch.Tensor:
    """float32(rs.normal(loc, scale, shape)) for a NumPy RandomState ``rs``, drawn on
    the device from rs's state (umapb_legacy_normal); ``rs`` itself is not advanced.
    ``parallel=False`` takes the one-CTA walk instead of the grid-wide path."""
    from mlx_vis_b200._nndescent.nndescent import state_words

    state = torch.from_numpy(state_words(rs.get_state())).to(device)
    out = torch.empty(shape, dtype=torch.float32, device=device)
    ws = workspace(query("umapb_legacy_normal_workspace", out.numel()), device) if parallel else None
    call("umapb_legacy_normal", ptr(state), out.numel(), float(loc), float(scale), ptr(out), ptr(ws),
         ws.numel() if ws is not None else 0, stream_handle())
    return out


def mt_jump_poly(b: int):
    """(coefficients, D): x^D mod phi for D = b * 65536 as a bool array of length
    19937 (coefficient of x^i at i), phi MT19937's characteristic polynomial; host
    code of the library, no GPU needed (umapb_mt_jump_poly)."""
    out = np.zeros(312, dtype=np.uint64)
    D = _i64(0)
    call("umapb_mt_jump_poly", int(b), out.ctypes.data, _c.byref(D))
    bits = np.unpackbits(out.view(np.uint8), bitorder="little")[:19937].astype(bool)
    return bits, int(D.value)


def set_wait_limit_ns(ns: int) -> None:
    """Time limit of the spectral power iteration's grid barrier (0: the 2 s default)."""
    call("umapb_set_wait_limit_ns", int(ns))


def spectral(rows, cols, vals, n_edges, n: int, dim: int, V0: torch.Tensor, noise: torch.Tensor,
             n_iter: int = 100, check: bool = False, fallback_seed=None, return_workspace: bool = False):
    """Spectral initial embedding (n, dim).  ``check`` synchronises and raises if
    the power iteration's grid barrier gave up.  With ``fallback_seed`` a failed
    power iteration is replaced on the device by the random start
    ``normal((n, dim), fallback_seed) * 0.01`` (umapb_spectral_fallback), with no
    synchronisation; the workspace (returned with ``return_workspace``) holds the
    status word that tells which one Y is."""
    V0 = _require(V0, torch.float32, 2, "V0")
    noise = _require(noise, torch.float32, 2, "noise")
    dev = V0.device
    e_cap = rows.numel()
    ws = workspace(query("umapb_spectral_workspace", n, dim, e_cap, n_iter), dev)
    Y = torch.empty((n, dim), dtype=torch.float32, device=dev)
    call("umapb_spectral", ptr(rows), ptr(cols), ptr(vals), ptr(n_edges), e_cap, n, dim, ptr(V0), int(n_iter),
         ptr(noise), ptr(Y), ptr(ws), ws.numel(), stream_handle())
    if fallback_seed is not None:
        call("umapb_spectral_fallback", ptr(ws), ptr(Y), n, dim, int(fallback_seed) & 0xFFFFFFFFFFFFFFFF,
             stream_handle())
    if check:
        read_status(ws)
    return (Y, ws) if return_workspace else Y


def status_word(ws: torch.Tensor) -> int:
    """The device status word at the start of a workspace (synchronises)."""
    return int(ws[:4].view(torch.int32).item())


class Layout:
    """Device state of one optimize_layout run (schedule + workspace)."""

    def __init__(self, rows, cols, vals, n_edges, n: int, dim: int, n_epochs: int):
        self.rows, self.cols, self.n_edges = rows, cols, n_edges
        self.n, self.dim, self.n_epochs = int(n), int(dim), int(n_epochs)
        self.e_cap = rows.numel()
        dev = rows.device
        self.ws = workspace(query("umapb_layout_workspace", self.n, self.dim, self.e_cap), dev)
        self.eps = torch.empty(max(self.e_cap, 1), dtype=torch.float32, device=dev)
        self.next = torch.empty(max(self.e_cap, 1), dtype=torch.float32, device=dev)
        call("umapb_layout_prepare", ptr(vals), ptr(n_edges), self.e_cap, self.n_epochs, ptr(self.eps),
             ptr(self.next), ptr(self.ws), self.ws.numel(), stream_handle())

    def epochs(self, Y: torch.Tensor, begin: int, end: int, a: float, b: float, learning_rate: float,
               neg_rate: int, seed: int, graph: bool = False):
        """Runs epochs [begin, end); with ``graph`` as one cached, updated CUDA graph."""
        call("umapb_layout_epochs_graph" if graph else "umapb_layout_epochs", ptr(Y), self.n, self.dim,
             ptr(self.rows), ptr(self.cols), ptr(self.eps),
             ptr(self.next), ptr(self.n_edges), self.e_cap, int(begin), int(end), self.n_epochs, float(a), float(b),
             float(learning_rate), int(neg_rate), int(seed) & 0xFFFFFFFFFFFFFFFF, ptr(self.ws), self.ws.numel(),
             stream_handle())

    def count_active(self, epoch: int) -> int:
        """Active edges in ``epoch`` for the current schedule state (synchronises)."""
        out = torch.zeros(1, dtype=torch.int64, device=self.rows.device)
        call("umapb_layout_count_active", ptr(self.next), ptr(self.n_edges), self.n, self.dim, self.e_cap,
             int(epoch), ptr(out), ptr(self.ws), self.ws.numel(), stream_handle())
        return int(out.item())

    def epoch_injected(self, Y: torch.Tensor, epoch: int, a: float, b: float, learning_rate: float, neg_rate: int,
                       neg_to: torch.Tensor):
        neg_to = _require(neg_to, torch.int32, 1, "neg_to")
        call("umapb_layout_epoch_injected", ptr(Y), self.n, self.dim, ptr(self.rows), ptr(self.cols),
             ptr(self.eps), ptr(self.next), ptr(self.n_edges), self.e_cap, int(epoch), self.n_epochs, float(a),
             float(b), float(learning_rate), int(neg_rate), ptr(neg_to), neg_to.numel(), ptr(self.ws),
             self.ws.numel(), stream_handle())


def _kp(k: int) -> int:
    return max(64, (int(k) + 63) // 64 * 64)


def split3(S: torch.Tensor, mu=None, transpose: bool = False, kp: int | None = None, out=None):
    """Split-precision operand rows of S (rows x cols, float32): S rows (K = cols) or,
    with ``transpose``, S columns (K = rows), mu subtracted per stored column.
    Returns (bf16 tensor (operand rows, 3 kp), kp); ``out``: a contiguous tensor of
    that shape to write into (a row block of a larger split, say)."""
    S = _require(S, torch.float32, 2, "S")
    rows, cols = S.shape
    kp = _kp(rows if transpose else cols) if kp is None else int(kp)
    shape = ((cols if transpose else rows), 3 * kp)
    if out is None:
        out = torch.empty(shape, dtype=torch.bfloat16, device=S.device)
    elif tuple(out.shape) != shape or out.dtype != torch.bfloat16 or not out.is_contiguous():
        raise ValueError(f"split3: out must be a contiguous bfloat16 tensor of shape {shape}")
    if mu is not None:
        mu = _require(mu, torch.float32, 1, "mu")
    call("umapb_split3", ptr(S), rows, cols, S.stride(0), ptr(mu), int(bool(transpose)), kp, ptr(out),
         stream_handle())
    return out, kp


SPLIT_SLICE_K = 1024  # K values per accumulator slice when ksplit is chosen automatically


def gemm_split3(A3: torch.Tensor, B3: torch.Tensor, kp: int, ksplit: int | None = None, scale: float = 1.0,
                status: torch.Tensor | None = None, out: torch.Tensor | None = None) -> torch.Tensor:
    """C = A B^T (M x N, float32) from split operands (FP32-level products on tcgen05).

    The tensor cores add the products of one accumulator in FP32; over a long K
    (a covariance over tens of thousands of rows, all products of a diagonal entry
    positive) that rounding grows with K, so by default the K range is cut into
    slices of at most 1024 values whose partial results are summed in FP64."""
    M, N = A3.shape[0], B3.shape[0]
    dev = A3.device
    if ksplit is None:
        ksplit = max(1, min(4096, -(-int(kp) // SPLIT_SLICE_K)))
    st = torch.zeros(1, dtype=torch.int32, device=dev) if status is None else status
    if out is not None:  # one slice straight into out (M x N, contiguous float32)
        if ksplit != 1 or scale != 1.0 or tuple(out.shape) != (M, N) or out.dtype != torch.float32 \
                or not out.is_contiguous():
            raise ValueError("gemm_split3: out needs ksplit 1, scale 1 and a contiguous float32 (M, N) tensor")
        call("umapb_gemm_split3", ptr(A3), ptr(B3), M, N, int(kp), 1, ptr(out), N, ptr(st), stream_handle())
        return out
    C = torch.empty((ksplit, M, N), dtype=torch.float32, device=dev)
    call("umapb_gemm_split3", ptr(A3), ptr(B3), M, N, int(kp), int(ksplit), ptr(C), N, ptr(st), stream_handle())
    if ksplit == 1 and scale == 1.0:
        return C[0]
    out = torch.empty((M, N), dtype=torch.float32, device=dev)
    call("umapb_sum_slices", ptr(C), int(ksplit), M * N, float(scale), ptr(out), stream_handle())
    return out


def matmul(A: torch.Tensor, B: torch.Tensor, A3=None) -> torch.Tensor:
    """A @ B for float32 A (M x K) and B (K x N) on the tensor cores with FP32-level
    error (umapb_split3 + umapb_gemm_split3).  ``A3``: A already split (split3(A))."""
    A3, kp = A3 if A3 is not None else split3(A)
    B3, _ = split3(B, transpose=True, kp=kp)
    return gemm_split3(A3, B3, kp)


def colmean(S: torch.Tensor) -> torch.Tensor:
    S = _require(S, torch.float32, 2, "S")
    rows, cols = S.shape
    ws = workspace(query("umapb_colmean_workspace", rows, cols), S.device)
    mean = torch.empty(cols, dtype=torch.float32, device=S.device)
    call("umapb_colmean", ptr(S), rows, cols, S.stride(0), ptr(mean), ptr(ws), ws.numel(), stream_handle())
    return mean


def sort_keys(keys: torch.Tensor) -> torch.Tensor:
    """Stable ascending order (int32) of a float32 vector (strided views allowed,
    e.g. one column of a row-major matrix)."""
    if not isinstance(keys, torch.Tensor) or not keys.is_cuda or keys.dtype != torch.float32 or keys.dim() != 1:
        raise ValueError("keys must be a 1-D float32 CUDA tensor")
    n = keys.numel()
    order = torch.empty(n, dtype=torch.int32, device=keys.device)
    ws = workspace(query("umapb_sort_keys_workspace", n), keys.device)
    call("umapb_sort_keys", _c.c_void_p(keys.data_ptr()), n, max(keys.stride(0), 1), ptr(order), ptr(ws), ws.numel(),
         stream_handle())
    return order


def exported_symbols() -> list[str]:
    return list(SIGNATURES)


def to_numpy(t: torch.Tensor) -> np.ndarray:
    return t.detach().cpu().numpy()
