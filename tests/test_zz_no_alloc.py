"""The allocation-free brute-force kNN entry point, umapb_knn_brute_noalloc.

It is there for callers that cannot give the library a device workspace:
cudaMalloc and cudaFree synchronise the whole device, they fail when another
framework's pooled allocator already holds the memory, and thin FFI bindings
may have no way to keep a device buffer alive between calls.  Its scratch is a
static device array inside the library, shared by every call, so the checks
here call it twice in a row (and after a call with a different shape) and
compare each result with the workspace entry point, umapb_knn_brute.

This file is collected last on purpose: a failure here leaves every other test
already run.
"""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def knn_noalloc(X: torch.Tensor, k: int, extra: int = 16, squared: bool = False):
    from mlx_vis_b200 import _lib

    n, d = X.shape
    idx = torch.empty((n, k), dtype=torch.int32, device=X.device)
    dist = torch.empty((n, k), dtype=torch.float32, device=X.device)
    status = torch.full((1,), -1, dtype=torch.int32, device=X.device)
    _lib.call("umapb_knn_brute_noalloc", _lib.ptr(X), n, d, k, extra, int(squared), _lib.ptr(idx), _lib.ptr(dist),
              _lib.ptr(status), _lib.stream_handle())
    torch.cuda.synchronize()
    return idx, dist, int(status.item())


def test_noalloc_matches_workspace_entry_point_on_consecutive_calls(gauss2000, proto1500):
    from mlx_vis_b200 import _lib

    Xg = torch.from_numpy(gauss2000).cuda()
    Xp = torch.from_numpy(proto1500).cuda()
    ref_g = _lib.knn_brute(Xg, 15)
    ref_p = _lib.knn_brute(Xp, 15)
    # a different shape first, so the shared scratch holds another call's data
    for X, (ref_idx, ref_dist) in [(Xp, ref_p), (Xg, ref_g), (Xg, ref_g)]:
        idx, dist, status = knn_noalloc(X, 15)
        assert status == 0
        assert torch.equal(idx, ref_idx)
        torch.testing.assert_close(dist, ref_dist, rtol=1e-6, atol=1e-6)


def test_noalloc_squared_distances_match():
    from mlx_vis_b200 import _lib

    X = torch.from_numpy(np.random.default_rng(1).normal(size=(3000, 40)).astype(np.float32)).cuda()
    ref_idx, ref_d2 = _lib.knn_brute(X, 10, squared=True)
    for _ in range(2):
        idx, d2, status = knn_noalloc(X, 10, squared=True)
        assert status == 0 and torch.equal(idx, ref_idx)
        torch.testing.assert_close(d2, ref_d2, rtol=1e-6, atol=1e-6)


def test_noalloc_serves_long_candidate_lists():
    """k + extra = 128 on 1000 rows: the candidate merge needs more than 48 KB of
    shared memory per block, which the allocation-free entry point raises per
    device like the workspace entry point."""
    from mlx_vis_b200 import _lib

    X = torch.from_numpy(np.random.default_rng(2).normal(size=(1000, 24)).astype(np.float32)).cuda()
    ref_idx, ref_dist = _lib.knn_brute(X, 112, extra=16)
    for _ in range(2):
        idx, dist, status = knn_noalloc(X, 112, extra=16)
        assert status == 0 and torch.equal(idx, ref_idx)
        torch.testing.assert_close(dist, ref_dist, rtol=1e-6, atol=1e-6)


def test_noalloc_rejects_requests_beyond_its_scratch():
    from mlx_vis_b200 import _lib

    X = torch.zeros((20000, 784), dtype=torch.float32, device="cuda")
    with pytest.raises(_lib.UmapB200Error, match="static array"):
        knn_noalloc(X, 15)
