"""Float64 reference of the warm-start encoder (test infrastructure).

The encoder has no counterpart in the reference (its closest idiom is the MMAE
MLP trained with AdamW, mlx_vis/_mmae/mmae.py:22-38, 258-281).  This module
computes its loss and gradients with torch float64 autograd on the CPU and one
AdamW step with ``torch.optim.AdamW``, so the library's hand-written forward,
backward and AdamW kernels can be checked.  ``bf16_like_gpu`` rounds the
operands the GPU keeps in BF16 (X, W1, W2, H1, H2 in the forward pass; dZ2 and
dZ1 in the backward pass, through straight-through rounding), which isolates
FP32-accumulation differences from the intended BF16 storage.
"""

from __future__ import annotations

import numpy as np
import torch


def _bf16(t: torch.Tensor) -> torch.Tensor:
    return t.to(torch.bfloat16).to(torch.float64)


class _RoundGrad(torch.autograd.Function):
    """Identity forward; rounds the incoming gradient to BF16 (the GPU stores dZ in BF16)."""

    @staticmethod
    def forward(ctx, x):
        return x.view_as(x)

    @staticmethod
    def backward(ctx, g):
        return _bf16(g)


def loss_and_grads(params: dict, X: np.ndarray, T: np.ndarray, bf16_like_gpu: bool = True):
    p = {k: torch.tensor(np.asarray(v, dtype=np.float64), requires_grad=True) for k, v in params.items()}
    x = torch.tensor(np.asarray(X, dtype=np.float64))
    t = torch.tensor(np.asarray(T, dtype=np.float64))
    gelu = torch.nn.functional.gelu
    if bf16_like_gpu:
        x = _bf16(x)
        w1 = p["W1"] + (_bf16(p["W1"]) - p["W1"]).detach()
        w2 = p["W2"] + (_bf16(p["W2"]) - p["W2"]).detach()
    else:
        w1, w2 = p["W1"], p["W2"]
    z1 = x @ w1.T + p["b1"]
    if bf16_like_gpu:
        z1 = _RoundGrad.apply(z1)
    h1 = gelu(z1)
    if bf16_like_gpu:
        h1 = h1 + (_bf16(h1) - h1).detach()
    z2 = h1 @ w2.T + p["b2"]
    if bf16_like_gpu:
        z2 = _RoundGrad.apply(z2)
    h2 = gelu(z2)
    if bf16_like_gpu:
        h2 = h2 + (_bf16(h2) - h2).detach()
    y = h2 @ p["W3"].T + p["b3"]
    loss = ((y - t) ** 2).sum(dim=1).mean()
    loss.backward()
    return float(loss), {k: v.grad.numpy() for k, v in p.items()}, y.detach().numpy()


def adamw_step(params: dict, grads: dict, lr=1e-3, betas=(0.9, 0.999), eps=1e-8, weight_decay=1e-2, steps=1):
    """``steps`` AdamW updates with the same gradients, float64; returns the new parameters."""
    p = {k: torch.nn.Parameter(torch.tensor(np.asarray(v, dtype=np.float64))) for k, v in params.items()}
    opt = torch.optim.AdamW(list(p.values()), lr=lr, betas=betas, eps=eps, weight_decay=weight_decay)
    for _ in range(steps):
        for k, v in p.items():
            v.grad = torch.tensor(np.asarray(grads[k], dtype=np.float64))
        opt.step()
    return {k: v.detach().numpy() for k, v in p.items()}
