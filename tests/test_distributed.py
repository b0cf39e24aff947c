"""Row-sharded brute-force kNN (mlx_vis_b200/_distributed.py) over world_size 2 and 3
gloo ranks on CPU: every rank computes its block of query rows (here with the
float64 oracle standing in for the GPU kernel), one all-gather assembles the
result, and every rank ends with the exact kNN of all rows."""

import os
import socket
import sys

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _oracle_block(X, k, begin, count):
    """Exact kNN (float64, ties by index) of rows [begin, begin + count)."""
    Xn = X.numpy().astype(np.float64)
    sq = np.sum(Xn * Xn, axis=1)
    rows = np.arange(begin, begin + count)
    d2 = sq[rows, None] + sq[None, :] - 2.0 * Xn[rows] @ Xn.T
    d2[np.arange(count), rows] = np.inf
    order = np.lexsort((np.broadcast_to(np.arange(len(Xn)), d2.shape), d2), axis=1)[:, :k]
    idx = torch.from_numpy(order.astype(np.int32))
    dst = torch.from_numpy(np.sqrt(np.maximum(np.take_along_axis(d2, order, axis=1), 0)).astype(np.float32))
    return idx, dst


def _rank(rank, world, port, q, n, d, k):
    sys.path.insert(0, REPO)
    from mlx_vis_b200._distributed import knn_brute_sharded

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        X = torch.from_numpy(np.random.default_rng(0).normal(size=(n, d)).astype(np.float32))
        idx, dst = knn_brute_sharded(X, k, block_knn=_oracle_block)
        dist.barrier()
        q.put((rank, idx.numpy(), dst.numpy()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,n", [(2, 301), (3, 100), (2, 3)])
def test_sharded_knn_assembles_every_row_on_every_rank(world, n):
    from mlx_vis_b200._distributed import row_blocks

    d, k = 7, 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q, n, d, k)) for r in range(world)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
    assert all(p.exitcode == 0 for p in procs)
    X = torch.from_numpy(np.random.default_rng(0).normal(size=(n, d)).astype(np.float32))
    want_i, want_d = _oracle_block(X, k, 0, n)
    for _, idx, dst in got:
        assert np.array_equal(idx, want_i.numpy())
        np.testing.assert_allclose(dst, want_d.numpy(), rtol=1e-6)
    assert sum(c for _, c in row_blocks(n, world)) == n


def test_row_blocks_cover_the_rows_in_order():
    from mlx_vis_b200._distributed import row_blocks

    for n in (1, 7, 70000):
        for world in (1, 2, 3, 8):
            b = row_blocks(n, world)
            assert len(b) == world and b[0][0] == 0
            assert all(b[i][0] + b[i][1] == b[i + 1][0] for i in range(world - 1))
            assert b[-1][0] + b[-1][1] == n
            assert max(c for _, c in b) - min(c for _, c in b) <= 1
