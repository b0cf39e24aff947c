"""CPU oracle for the UMAP hot path — TEST INFRASTRUCTURE ONLY.

A NumPy (float32 / float64) restatement of the reference's algorithms
(hanxiao/mlx-vis 0.7.0), each function citing the reference file:line it
follows.  It is the checker for the CUDA implementation in ``mlx_vis_b200``:
only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import it.  The product path never calls it.

Pinning: every restated function is checked against golden vectors produced by
running the reference's own unmodified modules on ``oracle/mlx_shim`` (a NumPy
implementation of the ``mlx.core`` subset they call), committed under
``tests/golden/`` together with the generating script ``make_golden.py``.

Modules
-------
knn        brute-force kNN: the reference's expanded float32 formula and an exact float64 version
nndescent  NNDescent graph construction (nndescent.py:34-486, 573-641)
fuzzy      smooth_knn_dist + symmetrisation + prune (umap.py:199-270)
spectral   spectral initialisation with injected draws (umap.py:298-357)
layout     epoch schedule and the synchronous SGD epoch (umap.py:359-449)
mlp        float64 autograd reference of the MLP encoder (new; no reference counterpart)
pipeline   the whole fit_transform on the host cores (CPU baseline of bench.py)
"""
