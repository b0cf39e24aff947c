"""Brute-force kNN sharded by query rows over the ranks of a torch.distributed group.

The reference's brute path walks the query rows in chunks against all points
(mlx_vis/_knn.py:58-79).  Here each rank (one process per GPU) takes one
contiguous block of query rows, computes their kNN against the full X that every
GPU holds (umapb_knn_brute_rows: tcgen05 distance tiles, fused top-(k+extra),
FP32 rerank), and one all-gather assembles the (n, k) result on every rank.
Only the (n, k) indices and distances cross NVLink (1.7 MB at 70,000 rows,
k = 15); no kernel reads another GPU's memory.
"""

from __future__ import annotations

import torch


def row_blocks(n: int, world: int) -> list[tuple[int, int]]:
    """(first row, row count) per rank: equal blocks, the first n % world ranks one
    row longer."""
    base, extra = divmod(int(n), int(world))
    out, begin = [], 0
    for r in range(world):
        count = base + (1 if r < extra else 0)
        out.append((begin, count))
        begin += count
    return out


def knn_brute_sharded(X: torch.Tensor, k: int, group=None, extra: int = 16, squared: bool = False,
                      block_knn=None):
    """kNN of every row of X (replicated on every rank) with the query rows split
    over the ranks of `group` (the default group; no group initialised: one rank).

    Returns (idx int32 (n, k), dist float32 (n, k)) on every rank, equal to
    umapb_knn_brute's result.  ``block_knn(X, k, begin, count)`` computes one
    block (default: the library's umapb_knn_brute_rows)."""
    import torch.distributed as dist

    n = X.shape[0]
    on = dist.is_available() and dist.is_initialized()
    world = dist.get_world_size(group) if on else 1
    rank = dist.get_rank(group) if on else 0
    if block_knn is None:
        from mlx_vis_b200 import _lib

        def block_knn(X_, k_, begin, count):
            return _lib.knn_brute_rows(X_, k_, begin, count, extra=extra, squared=squared)

    blocks = row_blocks(n, world)
    begin, count = blocks[rank]
    if count > 0:
        idx, dst = block_knn(X, k, begin, count)
    else:
        idx = torch.empty((0, k), dtype=torch.int32, device=X.device)
        dst = torch.empty((0, k), dtype=torch.float32, device=X.device)
    if world == 1:
        return idx, dst
    # all_gather needs equal shapes: pad every block to the longest
    m = max(c for _, c in blocks)
    pad_i = torch.zeros((m, k), dtype=torch.int32, device=idx.device)
    pad_d = torch.zeros((m, k), dtype=torch.float32, device=dst.device)
    pad_i[:count] = idx
    pad_d[:count] = dst
    gi = [torch.empty_like(pad_i) for _ in range(world)]
    gd = [torch.empty_like(pad_d) for _ in range(world)]
    dist.all_gather(gi, pad_i, group=group)
    dist.all_gather(gd, pad_d, group=group)
    out_i = torch.cat([gi[r][:c] for r, (_, c) in enumerate(blocks)])
    out_d = torch.cat([gd[r][:c] for r, (_, c) in enumerate(blocks)])
    return out_i, out_d
