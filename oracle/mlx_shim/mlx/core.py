"""A NumPy implementation of the subset of ``mlx.core`` that the reference's
UMAP hot path calls (``mlx_vis/_knn.py``, ``mlx_vis/_nndescent/nndescent.py``,
``mlx_vis/_umap/umap.py``).  Written from MLX's documented semantics:

* ``array`` is eager (``eval`` is a no-op, ``compile`` is the identity);
* Python floats become float32 and Python ints int32, float64 input arrays are
  narrowed to float32 (MLX has no float64 on the GPU);
* ``x.at[idx].add(v)`` / ``.multiply(v)`` are functional scatters in which
  duplicate indices accumulate (``np.add.at`` / ``np.multiply.at``);
* ``argsort`` returns uint32 indices; ties are ordered by position (a stable
  sort), which fixes an order MLX itself leaves unspecified;
* ``einsum`` on float16 inputs accumulates in float32 and rounds the result to
  float16, as the Metal kernels do;
* ``random`` draws come from a seeded NumPy PCG64 generator, so they are NOT
  MLX's bits.  Every draw is appended to ``random.log`` so that a caller can
  inject the same values into another implementation.

This is test infrastructure: the product never imports it.
"""

from __future__ import annotations

import builtins

import numpy as np

float32 = np.float32
float16 = np.float16
bfloat16 = np.float32  # not used on the UMAP path; placeholder type
int32 = np.int32
int64 = np.int64
uint32 = np.uint32
bool_ = np.bool_


class _Stream:
    def __init__(self, name):
        self.name = name


cpu = _Stream("cpu")
gpu = _Stream("gpu")


def _narrow(a: np.ndarray) -> np.ndarray:
    if a.dtype == np.float64:
        return a.astype(np.float32)
    if a.dtype == np.int64 and a.ndim == 0:
        return a.astype(np.int32)
    return a


class _At:
    def __init__(self, arr, idx):
        self._arr = arr
        self._idx = idx

    def add(self, v):
        out = np.array(self._arr, copy=True)
        np.add.at(out, _plain(self._idx), _plain(v))
        return out.view(array)

    def multiply(self, v):
        out = np.array(self._arr, copy=True)
        np.multiply.at(out, _plain(self._idx), _plain(v))
        return out.view(array)


class _AtIndexer:
    def __init__(self, arr):
        self._arr = arr

    def __getitem__(self, idx):
        return _At(self._arr, idx)


def _plain(x):
    if isinstance(x, tuple):
        return tuple(_plain(t) for t in x)
    if isinstance(x, np.ndarray):
        return x.view(np.ndarray)
    return x


class array(np.ndarray):
    """An eager MLX array backed by NumPy storage."""

    def __new__(cls, data=None, dtype=None):
        if isinstance(data, (bool, np.bool_)):
            a = np.asarray(data, dtype=np.bool_)
        elif isinstance(data, int) and dtype is None:
            a = np.asarray(data, dtype=np.int32)
        elif isinstance(data, float) and dtype is None:
            a = np.asarray(data, dtype=np.float32)
        else:
            a = np.asarray(_plain(data))
            if dtype is None:
                a = _narrow(a)
        if dtype is not None:
            a = a.astype(dtype)
        return np.array(a, copy=True).view(cls)

    @property
    def at(self):
        return _AtIndexer(self)

    def astype(self, dtype, *args, **kwargs):  # noqa: D401 - MLX signature
        return np.ndarray.astype(self, dtype).view(array)

    def __getitem__(self, idx):
        return np.ndarray.__getitem__(self, _plain(idx))


def _wrap(x):
    if isinstance(x, np.ndarray):
        return x.view(array)
    if isinstance(x, np.generic):
        return np.asarray(x).view(array)
    return x


def _arr(x):
    if isinstance(x, np.ndarray):
        return x.view(np.ndarray)
    if isinstance(x, float):
        return np.float32(x)
    if isinstance(x, bool):
        return np.bool_(x)
    if isinstance(x, int):
        return np.int32(x)
    return x


def eval(*args):  # noqa: A001 - MLX name
    return None


def compile(fn=None, **kwargs):  # noqa: A001 - MLX name
    if fn is None:
        return lambda f: f
    return fn


def zeros(shape, dtype=float32):
    return np.zeros(shape, dtype=dtype).view(array)


def ones(shape, dtype=float32):
    return np.ones(shape, dtype=dtype).view(array)


def full(shape, vals, dtype=None):
    if dtype is None:
        if isinstance(vals, float):
            dtype = float32
        elif isinstance(vals, bool):
            dtype = bool_
        elif isinstance(vals, int):
            dtype = int32
        else:
            dtype = _narrow(np.asarray(_plain(vals))).dtype
    return np.full(shape, _plain(vals), dtype=dtype).view(array)


def zeros_like(a):
    return np.zeros_like(_arr(a)).view(array)


def ones_like(a):
    return np.ones_like(_arr(a)).view(array)


def eye(n, m=None, k=0, dtype=float32):
    return np.eye(n, m, k, dtype=dtype).view(array)


def arange(*args, dtype=None):
    if dtype is None:
        dtype = float32 if builtins.any(isinstance(a, float) for a in args) else int32
    return np.arange(*args, dtype=dtype).view(array)


def sum(a, axis=None, keepdims=False):  # noqa: A001
    a = _arr(a)
    return _wrap(np.sum(a, axis=axis, keepdims=keepdims, dtype=a.dtype if a.dtype != np.bool_ else np.int32))


def mean(a, axis=None, keepdims=False):
    a = _arr(a)
    return _wrap(np.mean(a, axis=axis, keepdims=keepdims, dtype=a.dtype))


def min(a, axis=None, keepdims=False):  # noqa: A001
    return _wrap(np.min(_arr(a), axis=axis, keepdims=keepdims))


def max(a, axis=None, keepdims=False):  # noqa: A001
    return _wrap(np.max(_arr(a), axis=axis, keepdims=keepdims))


def all(a, axis=None, keepdims=False):  # noqa: A001
    return _wrap(np.all(_arr(a), axis=axis, keepdims=keepdims))


def any(a, axis=None, keepdims=False):  # noqa: A001
    return _wrap(np.any(_arr(a), axis=axis, keepdims=keepdims))


def maximum(a, b):
    return _wrap(np.maximum(_arr(a), _arr(b)))


def minimum(a, b):
    return _wrap(np.minimum(_arr(a), _arr(b)))


def where(c, a, b):
    a = _arr(a)
    b = _arr(b)
    out = np.where(_arr(c), a, b)
    # MLX keeps the array operand's dtype when the other operand is a scalar
    if isinstance(a, np.ndarray) and not isinstance(b, np.ndarray):
        out = out.astype(a.dtype)
    elif isinstance(b, np.ndarray) and not isinstance(a, np.ndarray):
        out = out.astype(b.dtype)
    return _wrap(out)


def exp(a):
    return _wrap(np.exp(_arr(a)))


def log(a):
    return _wrap(np.log(_arr(a)))


def sqrt(a):
    return _wrap(np.sqrt(_arr(a)))


def abs(a):  # noqa: A001
    return _wrap(np.abs(_arr(a)))


def power(a, b):
    return _wrap(np.power(_arr(a), _arr(b)))


def clip(a, a_min, a_max):
    return _wrap(np.clip(_arr(a), _arr(a_min), _arr(a_max)))


def square(a):
    return _wrap(np.square(_arr(a)))


def argsort(a, axis=-1):
    return _wrap(np.argsort(_arr(a), axis=axis, kind="stable").astype(np.uint32))


def sort(a, axis=-1):
    return _wrap(np.sort(_arr(a), axis=axis, kind="stable"))


def argpartition(a, kth, axis=-1):
    return _wrap(np.argpartition(_arr(a), kth, axis=axis).astype(np.uint32))


def take_along_axis(a, indices, axis):
    return _wrap(np.take_along_axis(_arr(a), _arr(indices).astype(np.int64), axis=axis))


def take(a, indices, axis=None):
    return _wrap(np.take(_arr(a), _arr(indices), axis=axis))


def concatenate(arrays, axis=0):
    return _wrap(np.concatenate([_arr(x) for x in arrays], axis=axis))


def stack(arrays, axis=0):
    return _wrap(np.stack([_arr(x) for x in arrays], axis=axis))


def broadcast_to(a, shape):
    return _wrap(np.ascontiguousarray(np.broadcast_to(_arr(a), shape)))


def reshape(a, shape):
    return _wrap(np.reshape(_arr(a), shape))


def cummax(a, axis=None, reverse=False, inclusive=True):
    a = _arr(a)
    if axis is None:
        a = a.reshape(-1)
        axis = 0
    if reverse:
        a = np.flip(a, axis)
    out = np.maximum.accumulate(a, axis=axis)
    if reverse:
        out = np.flip(out, axis)
    return _wrap(np.ascontiguousarray(out))


def cumsum(a, axis=None, reverse=False, inclusive=True):
    a = _arr(a)
    if axis is None:
        a = a.reshape(-1)
        axis = 0
    return _wrap(np.cumsum(a, axis=axis, dtype=a.dtype))


def einsum(subscripts, *operands):
    ops = [_arr(o) for o in operands]
    if all_half(ops):
        out = np.einsum(subscripts, *[o.astype(np.float32) for o in ops])
        return _wrap(out.astype(np.float16))
    return _wrap(np.einsum(subscripts, *ops))


def all_half(ops):
    for o in ops:
        if not (isinstance(o, np.ndarray) and o.dtype == np.float16):
            return False
    return True


def matmul(a, b):
    return _wrap(np.matmul(_arr(a), _arr(b)))


class _Random:
    """Seeded NumPy generator standing in for ``mlx.core.random``."""

    def __init__(self):
        self._gen = np.random.default_rng(0)
        self.log = []

    def seed(self, s):
        self._gen = np.random.default_rng(int(s))

    def normal(self, shape=(), dtype=float32, loc=0.0, scale=1.0, key=None):
        out = (self._gen.standard_normal(shape) * scale + loc).astype(dtype)
        self.log.append(("normal", out.copy()))
        return out.view(array)

    def uniform(self, low=0.0, high=1.0, shape=(), dtype=float32, key=None):
        out = self._gen.uniform(low, high, shape).astype(dtype)
        self.log.append(("uniform", out.copy()))
        return out.view(array)

    def randint(self, low, high, shape=(), dtype=int32, key=None):
        out = self._gen.integers(int(low), int(high), size=shape).astype(dtype)
        self.log.append(("randint", out.copy()))
        return out.view(array)


random = _Random()


class _Linalg:
    @staticmethod
    def eigh(a, UPLO="L", stream=None):
        w, v = np.linalg.eigh(_arr(a).astype(np.float64))
        return w.astype(np.float32).view(array), v.astype(np.float32).view(array)


linalg = _Linalg()
