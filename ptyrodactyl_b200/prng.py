"""Keys and draws of JAX's default random number generator, for the reference's
functions that take a ``PRNGKeyArray`` (``decompose_beam_to_modes``).

JAX (a dependency of the reference, pinned at 0.9.2, not installed here) draws with
the Threefry-2x32 block cipher, 20 rounds (Salmon, Moraes, Dror and Shaw, "Parallel
random numbers: as easy as 1, 2, 3", SC'11), in its "partitionable" counter layout,
the default since JAX 0.5. Restated here from those published rules:

* a key is two uint32 words; ``PRNGKey(seed)`` is (seed >> 32, seed & 0xffffffff);
* ``split(key, num)``: key i is the cipher block of the 64-bit counter i;
* 64-bit draws of a shape: element j is the cipher block of the counter j, high
  word first;
* ``uniform`` float64 on [lo, hi): the top 52 random bits as the mantissa of a
  number in [1, 2), minus 1, scaled, and clamped below at lo;
* ``normal`` float64: sqrt(2) erfinv(u), u uniform on [nextafter(-1, 0), 1).

XLA evaluates erfinv with its own polynomial; here it is SciPy's double-precision
erfinv, so a normal draw agrees with JAX's to a few units in the last place.
"""

from __future__ import annotations

from typing import Tuple

import numpy as np

Key = Tuple[int, int]

_ROTATIONS = ((13, 15, 26, 6), (17, 29, 16, 24))
_KS_PARITY = 0x1BD11BDA
_M32 = np.uint64(0xFFFFFFFF)


def _add(a: np.ndarray, b) -> np.ndarray:
    return ((a.astype(np.uint64) + np.uint64(b)) & _M32).astype(np.uint32) if np.isscalar(b) else \
        ((a.astype(np.uint64) + b.astype(np.uint64)) & _M32).astype(np.uint32)


def _rotl(x: np.ndarray, r: int) -> np.ndarray:
    return ((x << np.uint32(r)) | (x >> np.uint32(32 - r))).astype(np.uint32)


def threefry2x32(key: Key, c0: np.ndarray, c1: np.ndarray) -> Tuple[np.ndarray, np.ndarray]:
    """The 20-round Threefry-2x32 block of counters (c0, c1) (uint32 arrays) under
    ``key``: five groups of four add-rotate-xor rounds, the key schedule (k0, k1,
    k0 ^ k1 ^ 0x1BD11BDA) injected before the first group and after each, with the
    group number added to the second word."""
    ks = (int(key[0]) & 0xFFFFFFFF, int(key[1]) & 0xFFFFFFFF)
    ks = ks + ((ks[0] ^ ks[1] ^ _KS_PARITY) & 0xFFFFFFFF,)
    x0 = _add(np.asarray(c0, dtype=np.uint32), ks[0])
    x1 = _add(np.asarray(c1, dtype=np.uint32), ks[1])
    for group in range(5):
        for r in _ROTATIONS[group % 2]:
            x0 = _add(x0, x1)
            x1 = _rotl(x1, r) ^ x0
        x0 = _add(x0, ks[(group + 1) % 3])
        x1 = _add(x1, (ks[(group + 2) % 3] + group + 1) & 0xFFFFFFFF)
    return x0, x1


def prng_key(seed: int) -> Key:
    """jax.random.PRNGKey(seed)."""
    s = int(seed) & 0xFFFFFFFFFFFFFFFF
    return (s >> 32) & 0xFFFFFFFF, s & 0xFFFFFFFF


def as_key(key) -> Key:
    """A key given as a (hi, lo) pair or array of two uint32 words, or an int seed."""
    if isinstance(key, (int, np.integer)):
        return prng_key(int(key))
    words = np.asarray(key).reshape(-1)
    if words.size != 2:
        raise ValueError("a key is two uint32 words (or an int seed)")
    return int(words[0]) & 0xFFFFFFFF, int(words[1]) & 0xFFFFFFFF


def _counters(n: int) -> Tuple[np.ndarray, np.ndarray]:
    idx = np.arange(int(n), dtype=np.uint64)
    return (idx >> np.uint64(32)).astype(np.uint32), (idx & _M32).astype(np.uint32)


def split(key, num: int = 2) -> list:
    """jax.random.split(key, num)."""
    hi, lo = threefry2x32(as_key(key), *_counters(num))
    return [(int(a), int(b)) for a, b in zip(hi, lo)]


def bits64(key, shape) -> np.ndarray:
    """64-bit random words of ``shape``."""
    hi, lo = threefry2x32(as_key(key), *_counters(int(np.prod(shape))))
    return ((hi.astype(np.uint64) << np.uint64(32)) | lo.astype(np.uint64)).reshape(shape)


def uniform(key, shape, minval: float = 0.0, maxval: float = 1.0) -> np.ndarray:
    """jax.random.uniform(key, shape, float64, minval, maxval)."""
    one = np.array(1.0, dtype=np.float64).view(np.uint64)
    f = ((bits64(key, shape) >> np.uint64(12)) | one).view(np.float64) - 1.0
    return np.maximum(minval, f * (maxval - minval) + minval)


def normal(key, shape) -> np.ndarray:
    """jax.random.normal(key, shape, float64)."""
    from scipy.special import erfinv
    u = uniform(key, shape, float(np.nextafter(-1.0, 0.0)), 1.0)
    return np.sqrt(2.0) * erfinv(u)
