"""The C ABI: the library builds for sm_100a, loads without a GPU and exports
every function that include/umap_b200.h declares (no compute calls here)."""

import ctypes
import os
import re

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(REPO, "include", "umap_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(umapb_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    from mlx_vis_b200 import build

    path = build.build()
    return ctypes.CDLL(path)


def test_header_declares_the_api():
    names = declared_functions()
    assert "umapb_knn_brute" in names and "umapb_layout_epochs" in names and len(names) >= 10


def test_every_declared_symbol_is_exported(lib):
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_the_header():
    from mlx_vis_b200 import _lib

    assert sorted(_lib.SIGNATURES) == declared_functions()


def test_library_built_for_sm100a(lib):
    from mlx_vis_b200 import build

    assert "arch=compute_100a,code=sm_100a" in " ".join(build.NVCC_FLAGS)


def test_workspace_queries_and_argument_errors(lib):
    """Host-side validation runs without touching the GPU."""
    from mlx_vis_b200 import _lib

    _lib.load()
    nbytes = _lib.query("umapb_knn_brute_workspace", 20000, 784, 15, 16)
    # bf16 copy + norms + 2 candidate slots of 31 (score, index) pairs per row
    assert nbytes >= 20000 * 784 * 2 + 20000 * 31 * 8
    with pytest.raises(_lib.UmapB200Error, match="k <= n-1"):
        _lib.query("umapb_knn_brute_workspace", 10, 4, 10, 16)
    with pytest.raises(_lib.UmapB200Error, match="<= 128"):
        _lib.query("umapb_knn_brute_workspace", 1000, 4, 100, 40)
    assert _lib.query("umapb_fuzzy_workspace", 1000, 15) > 1000 * 15 * 8
    assert _lib.query("umapb_spectral_workspace", 100, 7, 1000, 100) > 0  # n_components up to 32
    with pytest.raises(_lib.UmapB200Error, match="dim <= 32"):
        _lib.query("umapb_spectral_workspace", 100, 33, 1000, 100)
    with pytest.raises(_lib.UmapB200Error, match="dim <= 32"):
        _lib.query("umapb_layout_workspace", 100, 33, 1000)
    assert _lib.load().umapb_abi_version() == 1


def test_python_signatures_have_the_header_arity():
    """Each ctypes argument list has as many entries as the C declaration has parameters."""
    from mlx_vis_b200 import _lib

    text = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    for name, params in re.findall(r"\b(umapb_[a-z0-9_]+)\s*\(([^)]*)\)\s*;", text):
        params = params.strip()
        n = 0 if params in ("", "void") else params.count(",") + 1
        assert len(_lib.SIGNATURES[name]) == n, (name, n, len(_lib.SIGNATURES[name]))
