"""NNDescent re-export (mirrors mlx_vis/nndescent.py)."""

from mlx_vis_b200._nndescent.nndescent import NNDescent

__all__ = ["NNDescent"]
