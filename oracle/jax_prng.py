"""Oracle support (test infrastructure only): JAX's default PRNG restated in NumPy.

The reference's golden-vector capture draws its input potential with
``jax.random.uniform(jax.random.PRNGKey(42), (32, 32, 2), dtype=float64) * 10``
(``tests/test_data/plan01_ug_capture.py:41-42``) and does not store it. JAX is a
third-party dependency absent here (pinned ``jax==0.9.2`` in the reference's
``uv.lock``), so this module restates the published algorithms it uses:

* Threefry-2x32 with 20 rounds (Salmon, Moraes, Dror, Shaw, "Parallel random
  numbers: as easy as 1, 2, 3", SC'11), the block cipher behind JAX's default
  ``threefry2x32`` key implementation;
* the seed -> key rule (high and low 32-bit words of the 64-bit seed);
* the counter layout of ``random_bits`` in both of JAX's modes
  ("partitionable", the default since JAX 0.5, and the original
  split-in-halves layout);
* ``uniform``'s mantissa-fill rule: keep the top ``nmant`` random bits, OR in the
  exponent of 1.0, reinterpret, subtract 1.

Only ``tests/golden/make_golden.py`` and the tests use this module.
"""

from __future__ import annotations

import numpy as np

_ROT = (13, 15, 26, 6, 17, 29, 16, 24)
_PARITY = np.uint32(0x1BD11BDA)


def _rotl(x: np.ndarray, r: int) -> np.ndarray:
    return ((x << np.uint32(r)) | (x >> np.uint32(32 - r))).astype(np.uint32)


def threefry2x32(key: tuple[int, int], x0: np.ndarray, x1: np.ndarray):
    """Threefry-2x32-20 of counter words (x0, x1) under a 2-word key.

    Five groups of four rounds; the key schedule is (k0, k1, k0^k1^parity)
    injected after every group with the group index added to the second word.
    """
    k0 = np.uint32(key[0])
    k1 = np.uint32(key[1])
    ks = (k0, k1, np.uint32(k0 ^ k1 ^ _PARITY))
    x0 = np.asarray(x0, dtype=np.uint32).copy()
    x1 = np.asarray(x1, dtype=np.uint32).copy()
    with np.errstate(over="ignore"):
        x0 = (x0 + ks[0]).astype(np.uint32)
        x1 = (x1 + ks[1]).astype(np.uint32)
        for group in range(5):
            rots = _ROT[0:4] if group % 2 == 0 else _ROT[4:8]
            for r in rots:
                x0 = (x0 + x1).astype(np.uint32)
                x1 = _rotl(x1, r)
                x1 = (x1 ^ x0).astype(np.uint32)
            x0 = (x0 + ks[(group + 1) % 3]).astype(np.uint32)
            x1 = (x1 + ks[(group + 2) % 3] + np.uint32(group + 1)).astype(np.uint32)
    return x0, x1


def prng_key(seed: int) -> tuple[int, int]:
    """``jax.random.PRNGKey(seed)`` for the threefry implementation."""
    seed = int(seed) & 0xFFFFFFFFFFFFFFFF
    return (seed >> 32) & 0xFFFFFFFF, seed & 0xFFFFFFFF


def random_bits64(key: tuple[int, int], shape, partitionable: bool = True) -> np.ndarray:
    """64-bit random words in JAX's layout for ``shape``."""
    size = int(np.prod(shape))
    if partitionable:
        idx = np.arange(size, dtype=np.uint64)
        hi = (idx >> np.uint64(32)).astype(np.uint32)
        lo = (idx & np.uint64(0xFFFFFFFF)).astype(np.uint32)
        b1, b2 = threefry2x32(key, hi, lo)
        bits = (b1.astype(np.uint64) << np.uint64(32)) | b2.astype(np.uint64)
        return bits.reshape(shape)
    # original layout: 2*size 32-bit words from a counter split into halves
    count = 2 * size
    ctr = np.arange(count, dtype=np.uint32)
    odd = count % 2
    if odd:
        ctr = np.concatenate([ctr, np.zeros(1, np.uint32)])
    half = ctr.size // 2
    y0, y1 = threefry2x32(key, ctr[:half], ctr[half:])
    words = np.concatenate([y0, y1])
    if odd:
        words = words[:-1]
    hi = words[:size].astype(np.uint64)
    lo = words[size:].astype(np.uint64)
    return ((hi << np.uint64(32)) | lo).reshape(shape)


def uniform_f64(key: tuple[int, int], shape, minval: float = 0.0, maxval: float = 1.0,
                partitionable: bool = True) -> np.ndarray:
    """``jax.random.uniform(key, shape, dtype=float64, minval, maxval)``."""
    bits = random_bits64(key, shape, partitionable)
    one_bits = np.array(1.0, dtype=np.float64).view(np.uint64)
    fbits = (bits >> np.uint64(64 - 52)) | one_bits
    floats = fbits.view(np.float64) - 1.0
    return np.maximum(minval, floats * (maxval - minval) + minval)
