"""UMAP re-export (mirrors mlx_vis/umap.py)."""

from mlx_vis_b200._umap.umap import UMAP

__all__ = ["UMAP"]
