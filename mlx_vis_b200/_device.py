"""Device selection and input conversion shared by the estimators."""

from __future__ import annotations

import numpy as np
import torch


def device() -> torch.device:
    if not torch.cuda.is_available():
        raise RuntimeError("mlx_vis_b200 needs a CUDA device (B200, sm_100a); none is visible")
    return torch.device("cuda", torch.cuda.current_device())


def to_device_f32(X, dev: torch.device | None = None) -> torch.Tensor:
    """numpy / array-like / torch input -> contiguous float32 (n, d) CUDA tensor.

    Host arrays go through pinned memory so the upload is one DMA."""
    dev = dev or device()
    if isinstance(X, torch.Tensor):
        t = X.detach()
        if t.dtype != torch.float32:
            t = t.float()
        return t.to(dev, non_blocking=True).contiguous()
    a = np.ascontiguousarray(np.asarray(X, dtype=np.float32))
    if a.ndim != 2:
        raise ValueError(f"expected a 2-D array (n_samples, n_features), got shape {a.shape}")
    host = torch.from_numpy(a)
    if a.nbytes >= (1 << 20):
        host = host.pin_memory()
    return host.to(dev, non_blocking=True)


def upload_async(X, dev: torch.device | None = None):
    """Like to_device_f32, but a host array is copied on a side stream: returns
    (tensor, event), and work that does not read the tensor may run on the current
    stream meanwhile; make the current stream wait on the event (None when X was
    already on the device) before the first kernel that reads it."""
    dev = dev or device()
    if isinstance(X, torch.Tensor) and X.is_cuda:
        return to_device_f32(X, dev), None
    if isinstance(X, torch.Tensor):
        host = X.detach()
        if host.dtype != torch.float32:
            host = host.float()
        host = host.contiguous()
    else:
        a = np.ascontiguousarray(np.asarray(X, dtype=np.float32))
        host = torch.from_numpy(a)
    if host.ndim != 2:
        raise ValueError(f"expected a 2-D array (n_samples, n_features), got shape {tuple(host.shape)}")
    if not host.is_pinned() and host.numel() * 4 >= (1 << 20):
        host = host.pin_memory()
    main = torch.cuda.current_stream(dev)
    Xd = torch.empty(host.shape, dtype=torch.float32, device=dev)
    side = copy_stream(dev)
    side.wait_stream(main)  # Xd's allocation is ordered on the current stream
    with torch.cuda.stream(side):
        Xd.copy_(host, non_blocking=True)
        done = torch.cuda.Event()
        done.record(side)
    Xd.record_stream(side)
    return Xd, done


def upload_blocks_async(X, dev: torch.device | None = None, blocks: int = 8):
    """Like upload_async, with the host rows copied in `blocks` row blocks: returns
    (tensor, done event, [(row_end, event), ...]) so that work on the first rows may
    start while the rest is still on its way (one block and no events when X is
    already on the device)."""
    dev = dev or device()
    if isinstance(X, torch.Tensor) and X.is_cuda:
        Xd = to_device_f32(X, dev)
        return Xd, None, []
    if isinstance(X, torch.Tensor):
        host = X.detach()
        if host.dtype != torch.float32:
            host = host.float()
        host = host.contiguous()
    else:
        host = torch.from_numpy(np.ascontiguousarray(np.asarray(X, dtype=np.float32)))
    if host.ndim != 2:
        raise ValueError(f"expected a 2-D array (n_samples, n_features), got shape {tuple(host.shape)}")
    if not host.is_pinned() and host.numel() * 4 >= (1 << 20):
        host = host.pin_memory()
    n = host.shape[0]
    main = torch.cuda.current_stream(dev)
    Xd = torch.empty(host.shape, dtype=torch.float32, device=dev)
    side = copy_stream(dev)
    side.wait_stream(main)  # Xd's allocation is ordered on the current stream
    marks = []
    step = max(1, -(-n // max(1, blocks)))
    with torch.cuda.stream(side):
        for r0 in range(0, n, step):
            r1 = min(n, r0 + step)
            Xd[r0:r1].copy_(host[r0:r1], non_blocking=True)
            e = torch.cuda.Event()
            e.record(side)
            marks.append((r1, e))
    Xd.record_stream(side)
    return Xd, marks[-1][1], marks


_copy_streams: dict = {}


def copy_stream(dev: torch.device) -> torch.cuda.Stream:
    """The side stream host uploads use on `dev`, made once per device (creating a
    stream per fit costs host time between fits)."""
    key = dev.index if dev.index is not None else torch.cuda.current_device()
    st = _copy_streams.get(key)
    if st is None:
        st = _copy_streams[key] = torch.cuda.Stream(device=dev)
    return st


def to_host(t: torch.Tensor) -> np.ndarray:
    return t.detach().cpu().numpy()
