"""mlx_vis_b200 — the UMAP hot path of mlx-vis (hanxiao/mlx-vis 0.7.0) rebuilt for
one NVIDIA B200 (sm_100a): PyTorch tensors on the host, hand-written CUDA kernels
in libumap_b200.so behind a C ABI (include/umap_b200.h), called through ctypes.

Drop-in names (mlx_vis/__init__.py:5-17): ``UMAP`` and ``NNDescent``; the shared
kNN plug point is ``mlx_vis_b200._knn.compute_knn``.
"""

__version__ = "0.1.0"

from mlx_vis_b200._umap.umap import UMAP
from mlx_vis_b200._nndescent.nndescent import NNDescent

__all__ = ["UMAP", "NNDescent"]
