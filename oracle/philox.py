"""Counter-based Philox4x32-10 random stream (test infrastructure).

This module is part of the ORACLE: a CPU checker for the CUDA path. Only the tests,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` may import it.

Philox4x32-10 is the counter-based generator of Salmon, Moraes, Dror and Shaw,
"Parallel random numbers: as easy as 1, 2, 3" (SC'11). The same function is written
in CUDA in ``hotspice_b200/csrc/hs_rng.cuh``; both sides must produce identical words.

The variate contract shared by the oracle and the CUDA kernels (one "call" = one
vectorised draw of the reference, e.g. one ``rng.random(size=k)``):

* key = (seed & 0xffffffff, seed >> 32)
* element ``e`` of call number ``c``: counter = (e, c & 0xffffffff, c >> 32, 0)
* ``u53 = ((w0 >> 5) * 2**26 + (w1 >> 6)) * 2**-53``  in [0, 1)

The reference draws from ``numpy.random`` / ``Generator`` (hotspice/core.py:83, 493,
527-538, 598-600, 666-671, 692, 698). Those draws are unseeded, so both the reference
(when generating golden fixtures) and this oracle are driven by :class:`PhiloxStream`.
"""
from __future__ import annotations

import numpy as np

_M0 = np.uint64(0xD2511F53)
_M1 = np.uint64(0xCD9E8D57)
_W0 = 0x9E3779B9
_W1 = 0xBB67AE85
_MASK = np.uint64(0xFFFFFFFF)


def philox4x32_10(c0, c1, c2, c3, k0: int, k1: int):
    """Vectorised Philox4x32 with 10 rounds. Counters are array-likes of uint32 values."""
    c0 = np.asarray(c0, dtype=np.uint64) & _MASK
    c1 = np.asarray(c1, dtype=np.uint64) & _MASK
    c2 = np.asarray(c2, dtype=np.uint64) & _MASK
    c3 = np.asarray(c3, dtype=np.uint64) & _MASK
    k0 = int(k0) & 0xFFFFFFFF
    k1 = int(k1) & 0xFFFFFFFF
    for _ in range(10):
        p0 = _M0 * c0
        p1 = _M1 * c2
        hi0, lo0 = p0 >> np.uint64(32), p0 & _MASK
        hi1, lo1 = p1 >> np.uint64(32), p1 & _MASK
        c0, c1, c2, c3 = (hi1 ^ c1 ^ np.uint64(k0)), lo1, (hi0 ^ c3 ^ np.uint64(k1)), lo0
        k0 = (k0 + _W0) & 0xFFFFFFFF
        k1 = (k1 + _W1) & 0xFFFFFFFF
    return (c0.astype(np.uint32), c1.astype(np.uint32), c2.astype(np.uint32), c3.astype(np.uint32))


def uniform53(seed: int, call: int, n: int) -> np.ndarray:
    """``n`` doubles in [0,1) for call number ``call`` (elements 0..n-1)."""
    e = np.arange(n, dtype=np.uint64)
    w0, w1, _, _ = philox4x32_10(e, call & 0xFFFFFFFF, (call >> 32) & 0xFFFFFFFF, 0,
                                 seed & 0xFFFFFFFF, (seed >> 32) & 0xFFFFFFFF)
    hi = (w0 >> np.uint32(5)).astype(np.float64)
    lo = (w1 >> np.uint32(6)).astype(np.float64)
    return (hi * 67108864.0 + lo) * (1.0 / 9007199254740992.0)


class PhiloxStream:
    """Drop-in for the subset of ``numpy.random`` / ``numpy.random.Generator`` that the
    reference hot path calls. Every method call consumes exactly one call number.

    Transforms (fixed here and mirrored by the CUDA kernels):
      random(size)            -> u
      exponential(scale,size) -> scale * (-log1p(-u))
      integers(lo, hi, size)  -> lo + floor(u * (hi - lo))
      randint                 -> integers
      choice(n, size)         -> floor(u * n)
      choice(n, size, replace=False) -> the first `size` of argsort(u over n elements, stable)
      permutation(n)          -> argsort(u over n elements, stable)
    """

    def __init__(self, seed: int, call: int = 0):
        self.seed = int(seed) & 0xFFFFFFFFFFFFFFFF
        self.call = int(call)
        self.log = []  # (method, n) per call, for debugging parity issues

    def _draw(self, shape, method):
        if shape is None:
            n, scalar = 1, True
        else:
            shape = (shape,) if np.isscalar(shape) else tuple(shape)
            n, scalar = int(np.prod(shape)) if len(shape) else 1, False
        u = uniform53(self.seed, self.call, n)
        self.log.append((method, n))
        self.call += 1
        if scalar:
            return float(u[0]), None
        return u.reshape(shape), shape

    # --- numpy.random.Generator / RandomState surface used by the reference ---
    def random(self, size=None):
        u, _ = self._draw(size, 'random')
        return u

    def random_sample(self, size=None):
        return self.random(size)

    def exponential(self, scale=1.0, size=None):
        u, _ = self._draw(size, 'exponential')
        with np.errstate(invalid='ignore', over='ignore'):
            return np.asarray(scale) * (-np.log1p(-np.asarray(u)))

    def integers(self, low, high=None, size=None, **kwargs):
        if high is None:
            low, high = 0, low
        u, _ = self._draw(size, 'integers')
        r = low + np.floor(np.asarray(u) * (high - low)).astype(np.int64)
        return int(r) if size is None else r

    def randint(self, low, high=None, size=None, dtype=int):
        return self.integers(low, high, size)

    def choice(self, a, size=None, replace=True, p=None):
        if not np.isscalar(a):
            raise NotImplementedError("PhiloxStream.choice only supports an integer population")
        if not replace:
            k = 1 if size is None else int(np.prod(size))
            if k > int(a):
                raise ValueError("Cannot take a larger sample than population when 'replace=False'")
            u, _ = self._draw(int(a), 'choice')
            r = np.argsort(np.atleast_1d(u), kind='stable')[:k]
            return int(r[0]) if size is None else r.reshape(size)
        u, _ = self._draw(size, 'choice')
        r = np.floor(np.asarray(u) * int(a)).astype(np.int64)
        return int(r) if size is None else r

    def permutation(self, x):
        if not np.isscalar(x):
            raise NotImplementedError("PhiloxStream.permutation only supports an integer length")
        u, _ = self._draw(int(x), 'permutation')
        return np.argsort(np.atleast_1d(u), kind='stable')

    def normal(self, *args, **kwargs):
        raise NotImplementedError("normal() is not on the hot path: pass E_B as an explicit array")

    def shuffle(self, x):
        raise NotImplementedError("shuffle() is only used by PoissonGrid, which is off by default")
