"""NumPy-backed stand-in for the ``mlx`` package (test infrastructure only).

MLX is not installable in this environment, so the reference's own UMAP /
NNDescent / kNN modules are executed against ``mlx.core`` as implemented in
``core.py`` next to this file.  Only ``tests/golden/make_golden.py`` (which
generates the committed golden fixtures) puts this directory on ``sys.path``.
"""
