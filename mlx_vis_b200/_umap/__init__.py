"""UMAP estimator package."""

from mlx_vis_b200._umap.umap import UMAP

__all__ = ["UMAP"]
