"""Restatement of the NumPy legacy-stream draws NNDescent's random start makes
(test infrastructure: the checker for the device generator ``umapb_nnd_random_start``).

mlx_vis/_nndescent/nndescent.py:47-57, 72-82 draws from NumPy's global
``RandomState``: ``randint(0, n - 1, (n, k), dtype=np.int32)``, then
``randn(d, 100)`` and ``randn(d, 300)`` when those are below d.  Those draws are:

* MT19937 (Matsumoto & Nishimura, ACM TOMACS 8(1), 1998): 624-word state,
  twist when the position reaches 624, tempered 32-bit outputs;
* bounded integers by masked rejection: with r = high - 1 - low and mask the
  smallest 2^m - 1 >= r, draw words until (w & mask) <= r (r == 0 draws nothing);
* standard normals by Marsaglia's polar method on 53-bit doubles
  ((a >> 5) * 2^26 + (b >> 6)) / 2^53 built from two words: x1, x2 uniform on
  (-1, 1), rejected unless 0 < r2 = x1^2 + x2^2 < 1, f = sqrt(-2 ln r2 / r2); the
  pair gives f*x2 now and caches f*x1 for the next call.

Pure Python and slow: for small sizes only.
"""

from __future__ import annotations

import math

import numpy as np

N, M = 624, 397
UPPER, LOWER, MATRIX_A = 0x80000000, 0x7FFFFFFF, 0x9908B0DF


def twist(mt: list[int]) -> list[int]:
    """One generation of the state, in the in-place order of the published algorithm."""
    mt = list(mt)
    for i in range(N):
        y = (mt[i] & UPPER) | (mt[(i + 1) % N] & LOWER)
        mt[i] = mt[(i + M) % N] ^ (y >> 1) ^ (MATRIX_A if y & 1 else 0)
    return mt


def temper(y: int) -> int:
    y ^= y >> 11
    y ^= (y << 7) & 0x9D2C5680
    y ^= (y << 15) & 0xEFC60000
    y ^= y >> 18
    return y & 0xFFFFFFFF


class Stream:
    """Word stream from a NumPy legacy state ('MT19937', key, pos, has_gauss, gauss)."""

    def __init__(self, state):
        _, key, pos, has_gauss, gauss = state[:5]
        self.key = [int(v) for v in key]
        self.pos = int(pos)
        self.has_gauss = int(has_gauss)
        self.gauss = float(gauss)

    def next32(self) -> int:
        if self.pos >= N:
            self.key = twist(self.key)
            self.pos = 0
        y = self.key[self.pos]
        self.pos += 1
        return temper(y)

    def next_double(self) -> float:
        a = self.next32() >> 5
        b = self.next32() >> 6
        return (a * 67108864.0 + b) / 9007199254740992.0

    def state(self):
        return ("MT19937", np.array(self.key, dtype=np.uint32), self.pos, self.has_gauss, self.gauss)


def gen_mask(r: int) -> int:
    m = r
    for s in (1, 2, 4, 8, 16):
        m |= m >> s
    return m


def randint(st: Stream, low: int, high: int, count: int) -> np.ndarray:
    r = high - 1 - low
    out = np.empty(count, dtype=np.int64)
    if r == 0:
        out[:] = low
        return out
    mask = gen_mask(r)
    for t in range(count):
        while True:
            v = st.next32() & mask
            if v <= r:
                break
        out[t] = low + v
    return out


def gauss(st: Stream) -> float:
    if st.has_gauss:
        st.has_gauss = 0
        g, st.gauss = st.gauss, 0.0
        return g
    while True:
        x1 = 2.0 * st.next_double() - 1.0
        x2 = 2.0 * st.next_double() - 1.0
        r2 = x1 * x1 + x2 * x2
        if 0.0 < r2 < 1.0:
            break
    f = math.sqrt(-2.0 * math.log(r2) / r2)
    st.gauss = f * x1
    st.has_gauss = 1
    return f * x2


def random_start(state, n: int, k: int, d: int):
    """(idx (n, k) int32, P or None, P2 or None, final state) of the reference's
    random start from the given legacy state (nndescent.py:54-56, 72-82)."""
    st = Stream(state)
    v = randint(st, 0, n - 1, n * k).reshape(n, k)
    rows = np.arange(n)[:, None]
    idx = np.where(v >= rows, v + 1, v).astype(np.int32)
    projs = []
    for pd in (min(100, d), min(300, d)):
        if pd < d:
            g = np.array([gauss(st) for _ in range(d * pd)], dtype=np.float64).reshape(d, pd)
            projs.append((g.astype(np.float32) / np.sqrt(pd)).astype(np.float32))
        else:
            projs.append(None)
    return idx, projs[0], projs[1], st.state()
