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
    # lists above 128 take the exact-tile path: split operand + one (R, n) tile
    assert _lib.query("umapb_knn_brute_workspace", 1000, 4, 100, 40) >= 1000 * 3 * 64 * 2 + 128 * 1000 * 4
    with pytest.raises(_lib.UmapB200Error, match="k must be <= 4096"):
        _lib.query("umapb_knn_brute_workspace", 10000, 4, 4097, 16)
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


def _raw_words(key, total):
    """x_0..x_{total-1}: the key, then x_n = x_{n-227} ^ mix(x_{n-624}, x_{n-623})."""
    import numpy as np

    x = np.zeros(total, dtype=np.uint32)
    x[:624] = key
    for base in range(624, total, 227):
        n = np.arange(base, min(total, base + 227))
        y = (x[n - 624] & np.uint32(0x80000000)) | (x[n - 623] & np.uint32(0x7FFFFFFF))
        x[n] = x[n - 227] ^ (y >> np.uint32(1)) ^ np.where(y & np.uint32(1), np.uint32(0x9908B0DF), np.uint32(0))
    return x


def test_mt_jump_polynomials_step_the_raw_stream(lib):
    """umapb_mt_jump_poly (host code): the words D = b * 65536 ahead of any position
    n >= 1 are the XOR of the words at n + i over the polynomial's set exponents i --
    the identity the device segments start from."""
    import numpy as np

    from mlx_vis_b200 import _lib
    from oracle.mt19937 import twist

    key = np.random.RandomState(11).get_state()[1]
    x = _raw_words(key, 5 * 65536 + 1300)
    g = [int(v) for v in key]
    for gen in range(1, 4):  # the vectorised recurrence is the published twist
        g = twist(g)
        assert np.array_equal(x[624 * gen:624 * (gen + 1)], np.array(g, dtype=np.uint32))
    w = np.arange(624)
    for b, base in ((1, 1), (1, 624), (2, 700), (5, 624)):
        bits, D = _lib.mt_jump_poly(b)
        assert D == b * 65536 and bits.sum() > 1000
        e = np.nonzero(bits)[0]
        got = np.bitwise_xor.reduce(x[base + e[:, None] + w[None, :]], axis=0)
        assert np.array_equal(got, x[base + D + w])
    for bad in (0, 1025):
        with pytest.raises(_lib.UmapB200Error):
            _lib.mt_jump_poly(bad)
