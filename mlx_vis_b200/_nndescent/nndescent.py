"""NNDescent on one B200 — drop-in for ``mlx_vis.NNDescent`` (mlx_vis/_nndescent/nndescent.py:14-403).

The control flow is the reference's, kept on the host:

* the same random draws from NumPy's global stream: ``np.random.seed``,
  ``randint(0, n-1, (n, k))`` shifted past self, then the two projections
  ``randn(d, 100)/sqrt(100)`` and ``randn(d, 300)/sqrt(300)`` (nndescent.py:47-82),
  so the random start and the projections are identical to the reference's.
  The draws are made on the device from the stream's state (MT19937, masked
  rejection, polar normals; random_start.cu) and the advanced state is handed
  back to NumPy, which leaves the global stream where the reference leaves it;
* per iteration mc_nn / j_nn from the update fraction (nndescent.py:100-101);
* full path while the update fraction is >= 0.5: iteration 0 in the 100-d
  projection, iteration 1 in the 300-d projection, FP16 distances in iterations
  1-4 with current distances recomputed, an FP32 recompute after iteration 4,
  reverse candidates while the fraction is >= 0.10 (nndescent.py:221-378);
* converging path below 0.5: only rows with a NEW neighbour, NEW neighbours
  first as sources, mc_new = max(3, int(k uf)), stored distances reused
  (nndescent.py:103-220);
* stop when the fraction of positional changes drops below delta (381-398).

Every data-parallel step runs in libumap_b200: the iterations in nndescent.cu,
the projections X @ P and X @ P2 as split-precision tcgen05 GEMMs with
FP32-level error (linalg.cu, gemm.cu), the locality order of the rows by the
library's radix sort.  One device-to-host read per iteration fetches the change
count that drives the control flow, as in the reference.
"""

from __future__ import annotations

import ctypes as _c
import os
import time

import numpy as np
import torch

from mlx_vis_b200 import _lib
from mlx_vis_b200._device import to_device_f32, to_host
from mlx_vis_b200._lib import call, ptr, query, stream_handle

# neighbours per row: up to 32 on the warp-per-row kernels with the blocked join,
# 33..100 on the block-per-row kernels (nnd_wide.cu)
MAX_K = 100
JOIN_MAX_K = 32


def iteration_params(update_frac: float, k: int, mc: int):
    """mc_nn, j_nn and the converging-path mc_new of nndescent.py:100-101, 107.

    The reference slices ``indices[:, :mc_new]``, so at most k sources are used;
    for k < 3 its floor of 3 sources makes its reshape fail, here it is clamped."""
    mc_nn = max(3, int(min(k, mc) * min(1.0, update_frac ** 0.5 * 3)))
    j_nn = max(k // 2, min(k, int(k * min(1.0, update_frac ** 0.5 * 3))))
    mc_conv = max(3, int(k * update_frac))
    return min(mc_nn, k), j_nn, min(mc_conv, k)


def state_words(state) -> np.ndarray:
    """np.random.get_state() as the uint32[628] buffer umapb_nnd_random_start reads."""
    name, key, pos, has_gauss, gauss = state[:5]
    if name != "MT19937":
        raise ValueError("NumPy's global stream is not MT19937")
    w = np.empty(628, dtype=np.uint32)
    w[:624] = key
    w[624], w[625] = pos, has_gauss
    w[626:] = np.array([gauss], dtype=np.float64).view(np.uint32)
    return w


def words_state(w: np.ndarray):
    """The inverse of state_words, for np.random.set_state."""
    w = np.asarray(w, dtype=np.uint32)
    return ("MT19937", w[:624].copy(), int(w[624]), int(w[625]), float(w[626:628].view(np.float64)[0]))


def random_start_device(n: int, k: int, d: int, random_state, dev, parallel: bool = True):
    """The reference's draws made on the device (umapb_nnd_random_start).

    Seeds NumPy's global stream like the reference, hands its state to the
    kernels and returns (idx, P, P2, state) with ``state`` the device buffer that
    holds the stream's state after the draws (give it back with
    ``np.random.set_state(words_state(state.cpu().numpy()))``).  ``parallel=False``
    takes the one-CTA walk instead of the grid-wide path."""
    if random_state is not None:
        np.random.seed(random_state)
    state = torch.from_numpy(state_words(np.random.get_state())).to(dev)
    pd1, pd2 = min(100, d), min(300, d)
    pd1, pd2 = (pd1 if pd1 < d else 0), (pd2 if pd2 < d else 0)
    idx = torch.empty((n, k), dtype=torch.int32, device=dev)
    P = torch.empty((d, pd1), dtype=torch.float32, device=dev) if pd1 else None
    P2 = torch.empty((d, pd2), dtype=torch.float32, device=dev) if pd2 else None
    ws = _lib.workspace(query("umapb_nnd_random_start_workspace", n, k, d, pd1, pd2), dev) if parallel else None
    call("umapb_nnd_random_start", ptr(state), n, k, d, ptr(idx), ptr(P), pd1, ptr(P2), pd2, ptr(ws),
         ws.numel() if ws is not None else 0, stream_handle())
    return idx, P, P2, state


def random_start(n: int, k: int, d: int, random_state):
    """The reference's draws on the host, in its order (nndescent.py:47-57, 72-82)."""
    if random_state is not None:
        np.random.seed(random_state)
    idx = np.random.randint(0, n - 1, (n, k), dtype=np.int32)
    i_vals = np.arange(n, dtype=np.int32)[:, None]
    idx = np.where(idx >= i_vals, idx + 1, idx).astype(np.int32)
    pd1, pd2 = min(100, d), min(300, d)
    P = (np.random.randn(d, pd1).astype(np.float32) / np.sqrt(pd1)).astype(np.float32) if pd1 < d else None
    P2 = (np.random.randn(d, pd2).astype(np.float32) / np.sqrt(pd2)).astype(np.float32) if pd2 < d else None
    return idx, P, P2


class NNDescent:
    """Approximate k-NN graph via NNDescent (constructor mirrors nndescent.py:17-32)."""

    def __init__(self, k: int = 15, n_iters: int = 20, max_candidates: int | None = None, delta: float = 0.015,
                 random_state: int | None = None, verbose: bool = False):
        self.k = k
        self.n_iters = n_iters
        self.max_candidates = max_candidates
        self.delta = delta
        self.random_state = random_state
        self.verbose = verbose
        self.neighbor_graph = None
        self.history_ = []
        self.profile_kernels = False  # record CUDA events around each iteration kernel

    def _events(self):
        if not self.profile_kernels:
            return None
        return (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))

    def build(self, X) -> tuple[np.ndarray, np.ndarray]:
        """Returns (indices int32 (n, k), Euclidean distances float32 (n, k)) on the host."""
        idx, dist = self.build_device(to_device_f32(X))
        self.neighbor_graph = (to_host(idx).astype(np.int32), to_host(dist).astype(np.float32))
        return self.neighbor_graph

    # ------------------------------------------------------------------
    def build_device(self, X: torch.Tensor, x_ready=None, x_blocks=None, while_first_iteration=None):
        """Device version of build: (idx int32, Euclidean dist float32) CUDA tensors.

        ``x_ready``: an event that X's upload records (see _device.upload_async);
        the random start, which does not read X, runs before the wait on it.
        ``x_blocks``: [(row_end, event), ...] of an upload in row blocks
        (_device.upload_blocks_async): the per-row preparation of a block then
        starts as soon as its rows have arrived.
        ``while_first_iteration``: a host function called once the first iteration's
        kernels are enqueued and before the host waits for its change count, so that
        its own host work (and the launches it makes on the current stream, which run
        after that iteration) overlaps the iteration on the device."""
        if not isinstance(X, torch.Tensor) or not X.is_cuda:
            X = to_device_f32(X)
            x_ready, x_blocks = None, None
        if x_blocks:
            x_ready = None
            if X.dtype != torch.float32 or not X.is_contiguous():
                raise ValueError("x_blocks needs a contiguous float32 X")
        elif x_ready is None:
            X = X.contiguous().float()
        n, d = X.shape
        if n < 2:
            raise ValueError("NNDescent needs at least 2 points")
        k = min(self.k, n - 1)
        if k > MAX_K:
            raise ValueError(f"NNDescent on the GPU supports k <= {MAX_K}")
        mc = self.max_candidates or k
        dev = X.device
        _lib.load()
        s = stream_handle()

        idx, P, P2, rng_state = random_start_device(n, k, d, self.random_state, dev)
        if x_ready is not None:
            torch.cuda.current_stream(dev).wait_event(x_ready)
            X = X.contiguous().float()
        dist = torch.empty((n, k), dtype=torch.float32, device=dev)

        # per-row preparation, one row block at a time: squared norms, the split of X
        # into BF16 parts, X @ P (iteration 0) and X @ P2 (iteration 1) on the tensor
        # cores with FP32-level error, and the FP16 rows of the FP16 iterations.  With
        # an upload in row blocks, a block starts once its rows are on the device.
        later = self.n_iters > 1
        sq = torch.empty(n, dtype=torch.float32, device=dev)
        X3 = P3 = P23 = kp = None
        X_low, sq_low = X, sq
        X300 = sq300 = X300h = None
        if P is not None:
            kp = _lib._kp(d)
            X3 = torch.empty((n, 3 * kp), dtype=torch.bfloat16, device=dev)
            P3, _ = _lib.split3(P, transpose=True, kp=kp)
            X_low = torch.empty((n, P.shape[1]), dtype=torch.float32, device=dev)
            sq_low = torch.empty(n, dtype=torch.float32, device=dev)
            if P2 is not None and later:
                P23, _ = _lib.split3(P2, transpose=True, kp=kp)
                X300 = torch.empty((n, P2.shape[1]), dtype=torch.float32, device=dev)
                sq300 = torch.empty(n, dtype=torch.float32, device=dev)
                ld300 = (P2.shape[1] + 7) // 8 * 8
                X300h = torch.empty((n, ld300), dtype=torch.float16, device=dev)
        ldh = (d + 7) // 8 * 8  # FP16 rows padded to 16-byte chunks
        Xh = torch.empty((n, ldh), dtype=torch.float16, device=dev) if later else None
        r0 = 0
        for r1, ready in (x_blocks or [(n, None)]):
            if ready is not None:
                torch.cuda.current_stream(dev).wait_event(ready)
            m = r1 - r0
            if m <= 0:
                continue
            Xb = X[r0:r1]
            call("umapb_nnd_sqnorms", ptr(Xb), m, d, 0, ptr(sq[r0:r1]), s)
            if P3 is not None:
                A3, _ = _lib.split3(Xb, kp=kp, out=X3[r0:r1])
                _lib.gemm_split3(A3, P3, kp, ksplit=1, out=X_low[r0:r1])
                call("umapb_nnd_sqnorms", ptr(X_low[r0:r1]), m, X_low.shape[1], 0, ptr(sq_low[r0:r1]), s)
                if X300 is not None:
                    _lib.gemm_split3(A3, P23, kp, ksplit=1, out=X300[r0:r1])
                    call("umapb_nnd_sqnorms", ptr(X300[r0:r1]), m, X300.shape[1], 0, ptr(sq300[r0:r1]), s)
                    call("umapb_nnd_to_half", ptr(X300[r0:r1]), m, X300.shape[1], X300h.shape[1], ptr(X300h[r0:r1]),
                         s)
            if Xh is not None:
                call("umapb_nnd_to_half", ptr(Xb), m, d, ldh, ptr(Xh[r0:r1]), s)
            if k <= JOIN_MAX_K:  # the random start's pairs whose later row is in this block
                call("umapb_nnd_gather_pairs", ptr(X), ptr(sq), n, d, ptr(idx), ptr(dist), k, r0, r1, s)
            r0 = r1
        X3 = P3 = P23 = None  # the split operands are not needed after the projections
        # the random start's FP32 distances, each row sorted (nndescent.py:59-65)
        if k <= JOIN_MAX_K:
            call("umapb_nnd_sort_rows", ptr(idx), ptr(dist), n, k, s)
        else:
            call("umapb_nnd_gather", ptr(X), ptr(sq), n, d, ptr(idx), ptr(dist), k, 1, s)

        # locality order of the rows (sorted by one random-projection coordinate):
        # rows and sources that run side by side then share most of their
        # candidate rows in the L2 cache; it changes no result
        order = _lib.sort_keys(X_low[:, 0]) if n > 1 else None
        rev = torch.empty((n, k), dtype=torch.int32, device=dev)
        rev_ws = _lib.workspace(query("umapb_nnd_reverse_workspace", n, k), dev)
        idx2 = torch.empty_like(idx)
        dist2 = torch.empty_like(dist)
        flags = torch.ones((n, k), dtype=torch.uint8, device=dev)
        flags2 = torch.empty_like(flags)
        # (changed, evals) counters of every iteration, zeroed once: an iteration
        # launches no fill and the host reads both with one copy
        counters = torch.zeros((max(self.n_iters, 1), 2), dtype=torch.int64, device=dev)
        # blocked nn-of-nn join (full path); UMAPB_NND_JOIN=0 computes every
        # candidate distance inside the row kernel instead
        join_on = os.environ.get("UMAPB_NND_JOIN", "1") != "0"
        nnbuf = curd = join_ws = None
        self.kernel_log_ = []  # (start event, end event, info) per iteration kernel when profile_kernels

        t0 = time.time()
        update_frac = 1.0
        self.history_ = []
        # FP32 distances of the current lists are due after the last FP16 iteration
        # (nndescent.py:376-378): a following full FP32 iteration takes them from its
        # join (every list position is a source there), anything else from a gather
        fp32_due = False
        # the loop's kernel arguments: device addresses looked up once per tensor (the
        # cache keeps each tensor alive, so an id is never reused for another one), and
        # the counters of iteration it at byte offset 16 it, so that the host work
        # between an iteration's count read and the next launches stays small
        cbase = counters.data_ptr()
        pcache = {}

        def P(t):
            if t is None:
                return _c.c_void_p(0)
            e = pcache.get(id(t))
            if e is None:
                e = pcache[id(t)] = (t, ptr(t))
            return e[1]

        for it in range(self.n_iters):
            mc_nn, j_nn, mc_conv = iteration_params(update_frac, k, mc)
            use_rev = update_frac >= 0.10
            changed_p = _c.c_void_p(cbase + 16 * it)  # counters[it, 0] and counters[it, 1]
            evals_p = _c.c_void_p(cbase + 16 * it + 8)
            ev = self._events()
            if update_frac < 0.5:
                # converging path: FP32, full dimension, stored distances
                if fp32_due:
                    call("umapb_nnd_gather", P(X), P(sq), n, d, P(idx), P(dist), k, 0, s)
                    fp32_due = False
                if use_rev:
                    call("umapb_nnd_reverse", P(idx), n, k, P(rev), P(rev_ws), rev_ws.numel(), s)
                # the nn-of-nn distances of the NEW-first sources from the blocked join
                join = join_on and k <= JOIN_MAX_K and mc_conv > 0 and j_nn > 0 and d % 4 == 0
                if join and nnbuf is None:
                    nnbuf = torch.empty(n * k * k, dtype=torch.float32, device=dev)
                    curd = torch.empty((n, k), dtype=torch.float32, device=dev)
                    join_ws = _lib.workspace(query("umapb_nnd_join_workspace", n, k, k), dev)
                ev[0].record() if ev else None
                if join:
                    call("umapb_nnd_join_new", P(X), P(sq), d, P(idx), P(flags), P(order), n, k, mc_conv,
                         j_nn, P(nnbuf), evals_p, P(join_ws), join_ws.numel(), s)
                call("umapb_nnd_iteration", P(X), P(sq), d, d, 0, P(idx), P(dist), P(flags),
                     P(rev if use_rev else None), P(order), P(nnbuf if join else None), P(None), n, k,
                     mc_conv, j_nn, 1, 0, P(idx2), P(dist2), P(flags2), changed_p, evals_p, s)
                ev[1].record() if ev else None
                info = dict(path="converging", mc_new=mc_conv, j_nn=j_nn, use_rev=use_rev, space=d, elem=4,
                            join=join)
            else:
                if it == 0:
                    Xd, sqd = X_low, sq_low
                elif it == 1 and X300 is not None:
                    Xd, sqd = X300, sq300
                else:
                    Xd, sqd = X, sq
                use_half = it in (1, 2, 3, 4)
                recompute = (it == 0) or use_half
                dd = Xd.shape[1]
                if fp32_due:
                    if not (Xd is X and not use_half and join_on and k <= JOIN_MAX_K and mc_nn == k
                            and d % 4 == 0):
                        call("umapb_nnd_gather", P(X), P(sq), n, d, P(idx), P(dist), k, 0, s)
                    else:
                        recompute = True  # the join's current-neighbour distances (curd)
                    fp32_due = False
                ldx = dd
                if use_half:
                    ldx = (dd + 7) // 8 * 8  # FP16 rows padded to 16-byte chunks
                    if Xd is X and Xh is not None:
                        src = Xh
                    elif Xd is X300:
                        src = X300h
                    else:
                        src = torch.empty((n, ldx), dtype=torch.float16, device=dev)
                        call("umapb_nnd_to_half", P(Xd), n, dd, ldx, P(src), s)
                else:
                    src = Xd
                join = join_on and k <= JOIN_MAX_K and mc_nn > 0 and (use_half or dd % 4 == 0)
                if join and nnbuf is None:
                    nnbuf = torch.empty(n * k * k, dtype=torch.float32, device=dev)
                    curd = torch.empty((n, k), dtype=torch.float32, device=dev)
                    join_ws = _lib.workspace(query("umapb_nnd_join_workspace", n, k, k), dev)
                # with every neighbour a source (mc_nn == k) the join's per-source
                # buckets are the reverse-candidate buckets: it writes rev itself
                rev_in_join = join and use_rev and mc_nn == k
                if use_rev and not rev_in_join:
                    call("umapb_nnd_reverse", P(idx), n, k, P(rev), P(rev_ws), rev_ws.numel(), s)
                ev[0].record() if ev else None
                if join:
                    call("umapb_nnd_join", P(src), P(sqd), dd, ldx, int(use_half), P(idx), P(order), n, k,
                         mc_nn, j_nn, P(nnbuf), P(curd), P(rev if rev_in_join else None), evals_p,
                         P(join_ws), join_ws.numel(), s)
                call("umapb_nnd_iteration", P(src), P(sqd), dd, ldx, int(use_half), P(idx), P(dist), P(None),
                     P(rev if use_rev else None), P(order), P(nnbuf if join else None),
                     P(curd if join else None), n, k, mc_nn, j_nn, 0, int(recompute), P(idx2),
                     P(dist2), P(flags2), changed_p, evals_p, s)
                ev[1].record() if ev else None
                if it == 4:  # FP32 recompute after the last FP16 iteration (nndescent.py:376-378)
                    fp32_due = True
                info = dict(path="full", mc_new=mc_nn, j_nn=j_nn, use_rev=use_rev, use_half=use_half, space=dd,
                            elem=2 if use_half else 4, join=join)
            if it == 0 and while_first_iteration is not None:
                while_first_iteration()
            n_changed, n_evals = counters[it].tolist()  # the one host read per iteration
            update_frac = n_changed / (n * k)
            idx, idx2 = idx2, idx
            dist, dist2 = dist2, dist
            flags, flags2 = flags2, flags
            info.update(it=it, changed=n_changed, evals=n_evals, n=n, k=k,
                        candidates=k + info["mc_new"] * j_nn + (k if use_rev else 0))
            if ev:
                self.kernel_log_.append((ev[0], ev[1], info))
            self.history_.append(info)
            if self.verbose:
                print(f"Iter {it + 1}/{self.n_iters}: {n_changed} updates ({update_frac:.4f}), "
                      f"{time.time() - t0:.2f}s")
            if update_frac < self.delta:
                if self.verbose:
                    print(f"Converged at iteration {it + 1}")
                break
        if fp32_due:  # the loop stopped after the last FP16 iteration
            call("umapb_nnd_gather", ptr(X), ptr(sq), n, d, ptr(idx), ptr(dist), k, 0, s)
        np.random.set_state(words_state(rng_state.cpu().numpy()))
        out = torch.empty_like(dist)
        _sqrt_into(dist, out)
        return idx, out


def _sqrt_into(d2: torch.Tensor, out: torch.Tensor) -> None:
    """Euclidean distances sqrt(max(d2, 0)) (nndescent.py:400) with the library kernel."""
    call("umapb_nnd_sqrt", ptr(d2), d2.numel(), ptr(out), stream_handle())

