"""Whole-fit CPU timing of the reference algorithm (test infrastructure, and the
CPU legs of bench.py).

The reference's own MLX CPU backend cannot be installed offline, so the CPU
figure is this oracle (a NumPy restatement of the reference's algorithm) on the
host cores.  A complete 70,000 x 784 fit of the reference code takes minutes on a
CPU (508 s for the reference's own modules on the NumPy mlx shim, 8 cores:
tests/golden/manifest.json, fixture c3_70k), more than a benchmark run can
spend, so ``FitSampler`` times every stage AT THE FULL SIZE but only a sample of
its work units, and scales each sample by an exact count of units:

  NNDescent (nndescent.py:34-403)  every iteration of the reference's own 70K run
      (its update log fixes each iteration's path, mc, j_nn and reverse
      candidates) on a block of rows of the 70K problem: candidate lists from the
      70K graph, reverse candidates of all 70K rows, row gathers of the
      iteration's space (100-d, 300-d FP16, 784-d), distances and the top-k;
      scaled by rows processed / block rows (all rows on the full path; on the
      converging path at most the changed entries of the previous iteration)
  fuzzy set (umap.py:199-270)      all 70K rows
  spectral init (umap.py:298-357)  the 70K graph with 5 and 10 power iterations:
      setup + per-iteration cost, extrapolated to 100 iterations
  layout (umap.py:389-449)         the host schedule of all 500 epochs, timed once;
      sampled epochs of the 70K graph scaled by positive-edge updates

Every figure is seconds of the full fit.
"""

from __future__ import annotations

import os
import time

import numpy as np

from oracle import fuzzy as ofz
from oracle import layout as olay
from oracle import nndescent as onnd
from oracle import spectral as ospec


def edge_updates(vals: np.ndarray, n_epochs: int) -> int:
    """Positive-edge updates of a whole optimize_layout run (umap.py:401-414)."""
    return int(sum(len(a) for a in olay.active_sets(vals, n_epochs)))


class FitSampler:
    """Sampled full-size timing of one fit (see the module docstring).

    X: (n, d) float32; ref_idx: the reference's NNDescent graph of X (n, k);
    ref_updates: the reference's per-iteration update counts for that build."""

    def __init__(self, X: np.ndarray, ref_idx: np.ndarray, ref_updates, n_epochs: int = 500, a: float = 1.5769,
                 b: float = 0.8951, seed: int = 0, block: int = 300, epochs_per_step: int = 2):
        self.X = np.ascontiguousarray(X, dtype=np.float32)
        n, d = self.X.shape
        self.n, self.d = n, d
        self.k = k = ref_idx.shape[1]
        self.n_epochs, self.a, self.b = n_epochs, a, b
        self.block, self.epochs_per_step = block, epochs_per_step
        self.step_no = 0
        self.sq = np.sum(self.X * self.X, axis=1, dtype=np.float32)
        self.idx = np.ascontiguousarray(ref_idx, dtype=np.int32)
        d2 = onnd.gather_d2(self.X, self.sq, self.idx)
        o = np.argsort(d2, axis=1, kind="stable")
        self.idx = np.take_along_axis(self.idx, o, axis=1)
        self.d2 = np.take_along_axis(d2, o, axis=1)
        # the iterations of the reference's own build: (update fraction entering it, changes before it)
        self.iters = []
        uf, prev = 1.0, n * k
        for u in ref_updates:
            self.iters.append((uf, prev))
            uf, prev = int(u) / (n * k), int(u)
        _, self.P, self.P2 = onnd.random_init(n, k, d, seed)
        self.graph = ofz.fuzzy_simplicial_set(self.idx, np.sqrt(self.d2), n_epochs, dtype=np.float32)[0]
        rows, cols, vals = self.graph
        t = time.perf_counter()
        self.sets = olay.active_sets(vals, n_epochs)  # the reference's host schedule (umap.py:407-414)
        self.t_schedule = time.perf_counter() - t
        self.updates_total = int(sum(len(s) for s in self.sets))
        self.nonempty = [e for e in range(n_epochs) if len(self.sets[e])]
        self.rng = np.random.default_rng(seed)
        self.Y0 = self.rng.uniform(0, 10, size=(n, 2)).astype(np.float32)
        self.threads = os.cpu_count()

    # ---- NNDescent --------------------------------------------------------
    def _dist(self, space, sq_s, rows, cols, half):
        """_gather_dists / _gather_dists_half (nndescent.py:573-641) for `rows`; with
        `half` the space is an FP16 array, converted once after the gather and the
        dot rounded to FP16, like the reference's FP16 einsum."""
        B = len(rows)
        f = cols.reshape(-1)
        A, C = space[rows], space[f]
        if half:
            A, C = A.astype(np.float32), C.astype(np.float32)
        dd = np.einsum("id,icd->ic", A, C.reshape(B, cols.shape[1], -1))
        if half:
            dd = dd.astype(np.float16).astype(np.float32)
        return np.maximum(sq_s[rows, None] + sq_s[f].reshape(cols.shape) - np.float32(2.0) * dd, np.float32(0))

    def _nnd_iteration(self, it: int, uf: float, rows: np.ndarray, Xd: np.ndarray, sqd: np.ndarray) -> None:
        """One iteration of the reference's row loop (nndescent.py:103-378) for `rows`."""
        k = self.k
        mc_nn, j_nn, mc_conv = onnd.iteration_params(uf, k, k)
        use_rev = uf >= 0.10
        if uf < 0.5:
            mc, use_half, recompute = mc_conv, False, False
        else:
            mc, use_half, recompute = mc_nn, it in (1, 2, 3, 4), it == 0 or it in (1, 2, 3, 4)
        B = len(rows)
        nc = self.idx[self.idx[rows, :mc].reshape(-1)].reshape(B, mc, k)[:, :, :j_nn].reshape(B, mc * j_nn)
        if use_rev:
            nc = np.concatenate([nc, self._rev[rows]], axis=1)
        new_d = self._dist(Xd, sqd, rows, nc, use_half)
        cur_d = self._dist(Xd, sqd, rows, self.idx[rows], use_half) if recompute else self.d2[rows]
        ac = np.concatenate([self.idx[rows], nc], axis=1)
        ad = np.concatenate([cur_d, new_d], axis=1)
        ad = np.where(ac == rows[:, None], onnd._BIG, ad)
        ri, _ = onnd.dedup_topk(ac, ad, k)
        if it == 4:  # the FP32 recompute after the last FP16 iteration (nndescent.py:376-378)
            self._dist(self.X, self.sq, rows, ri, False)

    def nndescent_s(self) -> float:
        n, k, B = self.n, self.k, self.block
        start = (self.step_no * 7919) % max(n - B, 1)
        rows = np.arange(start, start + B, dtype=np.int32)
        t = time.perf_counter()
        idx0, _, _ = onnd.random_init(n, k, self.d, 0)
        X_low = self.X @ self.P if self.P is not None else self.X
        sq_low = np.sum(X_low * X_low, axis=1, dtype=np.float32)
        t_total = time.perf_counter() - t
        t = time.perf_counter()  # the random graph's distances and initial sort (nndescent.py:59-65)
        d0 = self._dist(self.X, self.sq, rows, idx0[rows], False)
        np.argsort(d0, axis=1, kind="stable")
        t_total += (time.perf_counter() - t) * n / B
        spaces = {}
        for it, (uf, prev) in enumerate(self.iters):
            t = time.perf_counter()
            self._rev = onnd.reverse_candidates(self.idx) if uf >= 0.10 else None
            half = uf >= 0.5 and it in (1, 2, 3, 4)
            if uf >= 0.5:
                if it == 0:
                    Xd, sqd = X_low, sq_low
                elif it == 1 and self.P2 is not None:
                    X300 = self.X @ self.P2
                    spaces[300] = (X300, np.sum(X300 * X300, axis=1, dtype=np.float32))
                    Xd, sqd = spaces[300]
                else:
                    Xd, sqd = self.X, self.sq
                R = n
            else:
                Xd, sqd = self.X, self.sq
                R = min(n, prev)  # rows with a NEW neighbour: at most the entries changed before
            if half:  # the FP16 copy of the iteration's space, made at full size
                Xd = Xd.astype(np.float16)
            t_fixed = time.perf_counter() - t
            t = time.perf_counter()
            self._nnd_iteration(it, uf, rows, Xd, sqd)
            t_block = time.perf_counter() - t
            t_total += t_fixed + t_block * R / B
        return t_total

    # ---- the other stages -------------------------------------------------
    def fuzzy_s(self) -> float:
        t = time.perf_counter()
        ofz.fuzzy_simplicial_set(self.idx, np.sqrt(self.d2), self.n_epochs, dtype=np.float32)
        return time.perf_counter() - t

    def spectral_s(self) -> float:
        rows, cols, vals = self.graph
        V0 = self.rng.standard_normal((self.n, 3)).astype(np.float32)
        ts = []
        for it in (5, 10):
            t = time.perf_counter()
            ospec.spectral_init(rows, cols, vals, self.n, V0, 0, n_iter=it, dtype=np.float32)
            ts.append(time.perf_counter() - t)
        per_iter = max(ts[1] - ts[0], 0.0) / 5
        setup = max(ts[0] - 5 * per_iter, 0.0)
        return setup + 100 * per_iter

    def layout_s(self) -> float:
        rows, cols, vals = self.graph
        rows = np.asarray(rows, dtype=np.int64)
        cols = np.asarray(cols, dtype=np.int64)
        m = len(self.nonempty)
        pick = [self.nonempty[(self.step_no * 37 + j * (m // self.epochs_per_step + 1)) % m]
                for j in range(self.epochs_per_step)]
        t_ep, upd = 0.0, 0
        for e in pick:
            act = self.sets[e]
            ef, et = rows[act], cols[act]
            n_neg = 5 * len(act)
            t = time.perf_counter()
            neg_to = self.rng.integers(0, self.n, n_neg)
            olay.sgd_epoch(self.Y0, ef, et, ef[np.arange(n_neg) % len(act)], neg_to,
                           1.0 - e / self.n_epochs, self.a, self.b, dtype=np.float32)
            t_ep += time.perf_counter() - t
            upd += len(act)
        return self.t_schedule + t_ep * self.updates_total / max(upd, 1)

    def step(self) -> dict:
        """One sampled full-size fit: estimated seconds per stage and in total."""
        out = {"knn": self.nndescent_s(), "fuzzy": self.fuzzy_s(), "init": self.spectral_s(),
               "layout": self.layout_s()}
        out["fit"] = sum(out.values())
        self.step_no += 1
        return out

    def describe(self) -> str:
        return (f"{self.n} x {self.d} rows at full size: NNDescent's {len(self.iters)} iterations (the reference's "
                f"own 70K update log) on {self.block}-row blocks scaled by rows processed, the fuzzy set on all "
                f"rows, spectral init from 5 and 10 power iterations extrapolated to 100, the 500-epoch schedule "
                f"timed in full and {self.epochs_per_step} sampled epochs scaled by {self.updates_total} "
                f"positive-edge updates")
