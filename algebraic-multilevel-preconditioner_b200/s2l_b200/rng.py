"""Seeded random numbers that match the reference's right-hand sides bit for bit.

The reference draws its random right-hand side with ``std::mt19937_64(seed)`` and
``std::uniform_real_distribution<double>(-1, 1)`` in the original (unpermuted) ordering
(``src/partition/domain_decomposer.cpp:158-164``), and the bubble centres with the same
engine (``include/utils/bubble_field.hpp:64-72``).  This module restates the published
MT19937-64 generator (Matsumoto & Nishimura, 2004) with a vectorised twist, and the
libstdc++ mapping of a 64-bit draw to ``[a, b)``: ``u = double(draw) / 2**64`` (clamped below
1), ``a + u * (b - a)``.
"""
from __future__ import annotations

import numpy as np

_NN = 312
_MM = 156
_MATRIX_A = np.uint64(0xB5026F5AA96619E9)
_UM = np.uint64(0xFFFFFFFF80000000)
_LM = np.uint64(0x7FFFFFFF)


class MT19937_64:
    """MT19937-64 engine with the seeding of ``std::mt19937_64(seed)``."""

    def __init__(self, seed: int = 5489):
        mt = np.zeros(_NN, dtype=np.uint64)
        mask = (1 << 64) - 1
        v = seed & mask
        mt[0] = v
        for i in range(1, _NN):
            v = (6364136223846793005 * (v ^ (v >> 62)) + i) & mask
            mt[i] = v
        self._mt = mt
        self._buf = np.empty(0, dtype=np.uint64)
        self._pos = 0

    def _twist(self) -> None:
        mt = self._mt
        one = np.uint64(1)
        zero = np.uint64(0)
        # i in [0, NN-MM): reads mt[i+1] and mt[i+MM], all still old.
        i0 = np.arange(0, _NN - _MM)
        x = (mt[i0] & _UM) | (mt[i0 + 1] & _LM)
        mt[i0] = mt[i0 + _MM] ^ (x >> one) ^ np.where((x & one) == one, _MATRIX_A, zero)
        # i in [NN-MM, NN-1): reads mt[i+1] (old) and mt[i+MM-NN] (new, from the first block).
        i1 = np.arange(_NN - _MM, _NN - 1)
        x = (mt[i1] & _UM) | (mt[i1 + 1] & _LM)
        mt[i1] = mt[i1 + (_MM - _NN)] ^ (x >> one) ^ np.where((x & one) == one, _MATRIX_A, zero)
        # last element wraps to mt[0] (new).
        x = (mt[_NN - 1] & _UM) | (mt[0] & _LM)
        mt[_NN - 1] = mt[_MM - 1] ^ (x >> one) ^ (_MATRIX_A if (int(x) & 1) else zero)
        # tempering
        y = mt.copy()
        y ^= (y >> np.uint64(29)) & np.uint64(0x5555555555555555)
        y ^= (y << np.uint64(17)) & np.uint64(0x71D67FFFEDA60000)
        y ^= (y << np.uint64(37)) & np.uint64(0xFFF7EEE000000000)
        y ^= y >> np.uint64(43)
        self._buf = y
        self._pos = 0

    def draws(self, count: int) -> np.ndarray:
        """The next ``count`` 64-bit outputs of the engine."""
        out = np.empty(count, dtype=np.uint64)
        k = 0
        while k < count:
            if self._pos >= _NN:
                self._twist()
            if self._buf.size == 0:
                self._twist()
            take = min(count - k, _NN - self._pos)
            out[k:k + take] = self._buf[self._pos:self._pos + take]
            self._pos += take
            k += take
        return out

    def uniform(self, count: int, a: float = 0.0, b: float = 1.0) -> np.ndarray:
        """``std::uniform_real_distribution<double>(a, b)`` applied ``count`` times (libstdc++)."""
        u = self.draws(count).astype(np.float64) / 18446744073709551616.0
        u = np.where(u >= 1.0, np.nextafter(1.0, 0.0), u)
        return u * (b - a) + a


def random_rhs(n: int, seed: int) -> np.ndarray:
    """U[-1, 1] right-hand side in the original ordering, as the reference draws it."""
    return MT19937_64(seed).uniform(n, -1.0, 1.0)


_M32 = 0xFFFFFFFF


def seed_seq_generate(seeds, count: int) -> list:
    """``std::seed_seq(seeds).generate()`` of ``count`` 32-bit words: the algorithm the C++ standard
    specifies for ``seed_seq::generate`` ([rand.util.seedseq]), restated over Python integers."""
    v = [int(s) & _M32 for s in seeds]
    s, n = len(v), int(count)
    if n == 0:
        return []
    b = [0x8B8B8B8B] * n
    t = 11 if n >= 623 else 7 if n >= 68 else 5 if n >= 39 else 3 if n >= 7 else (n - 1) // 2
    p = (n - t) // 2
    q = p + t
    m = max(s + 1, n)

    def mix(x):
        return x ^ (x >> 27)

    for k in range(m):
        r1 = (1664525 * mix(b[k % n] ^ b[(k + p) % n] ^ b[(k - 1) % n])) & _M32
        if k == 0:
            r2 = r1 + s
        elif k <= s:
            r2 = r1 + k % n + v[k - 1]
        else:
            r2 = r1 + k % n
        r2 &= _M32
        b[(k + p) % n] = (b[(k + p) % n] + r1) & _M32
        b[(k + q) % n] = (b[(k + q) % n] + r2) & _M32
        b[k % n] = r2
    for k in range(m, m + n):
        r3 = (1566083941 * mix((b[k % n] + b[(k + p) % n] + b[(k - 1) % n]) & _M32)) & _M32
        r4 = (r3 - k % n) & _M32
        b[(k + p) % n] ^= r3
        b[(k + q) % n] ^= r4
        b[k % n] = r4
    return b


def mt19937_64_from_seed_seq(seeds) -> MT19937_64:
    """``std::mt19937_64(std::seed_seq{seeds...})``: 2 words of the sequence per 64-bit state word
    (low word first); an all-zero state (top 33 bits of the first word included) becomes 2^63."""
    words = seed_seq_generate(seeds, 2 * _NN)
    st = [(words[2 * i] | (words[2 * i + 1] << 32)) for i in range(_NN)]
    if (st[0] & int(_UM)) == 0 and not any(st[1:]):
        st[0] = 1 << 63
    eng = MT19937_64(0)
    eng._mt = np.asarray(st, dtype=np.uint64)
    eng._buf = np.empty(0, dtype=np.uint64)
    eng._pos = 0
    return eng


def random_rhs_step(n: int, seed: int, step: int, corrector: int) -> np.ndarray:
    """U[-1, 1] right-hand side of solve (step, corrector) of a sequence, original ordering: the
    reference's ``randomRhs`` (``src/solver/time_loop.cpp:31-43``), an ``std::mt19937_64`` seeded
    with ``std::seed_seq{seed, step, corrector, 0x5eed}``."""
    eng = mt19937_64_from_seed_seq([int(seed) & _M32, int(step) & _M32, int(corrector) & _M32, 0x5EED])
    return eng.uniform(n, -1.0, 1.0)
