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
  exponent of 1.0, reinterpret, subtract 1;
* ``split`` in the partitionable ("fold-like") layout: key i is the Threefry block of
  the counter (0, i) under the parent key;
* ``normal``: ``sqrt(2) * erf_inv(u)`` with ``u`` uniform on
  [nextafter(-1, 0), 1). XLA evaluates ``erf_inv`` with its own polynomial; here the
  inverse error function is computed to full double precision by Halley's method
  (so the draws agree with JAX's to a few units in the last place).

Only ``tests/golden/make_golden.py`` and the tests use this module.
"""

from __future__ import annotations

import math

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


def split(key: tuple[int, int], num: int = 2) -> list[tuple[int, int]]:
    """``jax.random.split(key, num)`` (partitionable layout): key i = Threefry-2x32 of
    the 64-bit counter i, as (high, low) words, under ``key``."""
    idx = np.arange(int(num), dtype=np.uint64)
    b1, b2 = threefry2x32(key, (idx >> np.uint64(32)).astype(np.uint32),
                          (idx & np.uint64(0xFFFFFFFF)).astype(np.uint32))
    return [(int(a), int(b)) for a, b in zip(b1, b2)]


def erfinv(y: float) -> float:
    """Inverse error function in double precision.

    Starting value: Winitzki's closed-form approximation (S. Winitzki, "A handy
    approximation for the error function and its inverse", 2008; a = 0.147, relative
    error ~2e-3). Refinement: Halley's method on f(x) = erf(x) - y, with
    f' = 2/sqrt(pi) exp(-x^2) and f'' = -2 x f', written through erfc in the tails so
    that 1 - |y| keeps its precision; three steps reach rounding level.
    """
    y = float(y)
    if y <= -1.0:
        return -math.inf
    if y >= 1.0:
        return math.inf
    if y == 0.0:
        return 0.0
    a = 0.147
    ln = math.log1p(-y * y)
    t = 2.0 / (math.pi * a) + 0.5 * ln
    x = math.copysign(math.sqrt(math.sqrt(t * t - ln / a) - t), y)
    ay = abs(y)
    for _ in range(4):
        if ay > 0.5:  # f = sign(y) (1 - |y| - erfc(|x|)) without cancellation
            f = ((1.0 - ay) - math.erfc(abs(x))) * (1.0 if y > 0 else -1.0)
        else:
            f = math.erf(x) - y
        d = 2.0 / math.sqrt(math.pi) * math.exp(-x * x)
        if d == 0.0:
            break
        step = f / d
        x = x - step / (1.0 + x * step)  # Halley: f'' / f' = -2 x
    return x


def normal_f64(key: tuple[int, int], shape) -> np.ndarray:
    """``jax.random.normal(key, shape, dtype=float64)``."""
    lo = np.nextafter(np.float64(-1.0), np.float64(0.0))
    u = uniform_f64(key, shape, minval=float(lo), maxval=1.0)
    return np.sqrt(np.float64(2.0)) * np.vectorize(erfinv, otypes=[np.float64])(u)
