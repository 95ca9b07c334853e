"""Host-side JAX key arithmetic (threefry2x32, partitionable layout).

Used only for key bookkeeping on the host (seeding runs, deriving the
replica-exchange key chain); every random number the walk consumes is drawn
on the device by the CUDA library from the same streams.  Keys are
``uint32[2]`` arrays holding ``jax.random.key_data`` words.

Semantics restated from JAX's public PRNG design (threefry2x32-20 of Salmon
et al., SC'11; ``split(key, n)[i] == fold_in(key, i) == hash(key, (0, i))``
under ``jax_threefry_partitionable=True``).
"""

from __future__ import annotations

import numpy as np

_ROT = (13, 15, 26, 6, 17, 29, 16, 24)


def _rotl(x: np.ndarray, r: int) -> np.ndarray:
    return (x << np.uint32(r)) | (x >> np.uint32(32 - r))


def threefry2x32(k0, k1, c0, c1):
    """Vectorised threefry2x32 with 20 rounds over uint32 arrays."""
    with np.errstate(over="ignore"):
        k0 = np.asarray(k0, np.uint32)
        k1 = np.asarray(k1, np.uint32)
        ks = (k0, k1, np.uint32(0x1BD11BDA) ^ k0 ^ k1)
        x0 = np.asarray(c0, np.uint32) + ks[0]
        x1 = np.asarray(c1, np.uint32) + ks[1]
        for r in range(20):
            x0 = x0 + x1
            x1 = _rotl(x1, _ROT[r % 8])
            x1 = x1 ^ x0
            if r % 4 == 3:
                s = r // 4 + 1
                x0 = x0 + ks[s % 3]
                x1 = x1 + ks[(s + 1) % 3] + np.uint32(s)
    return x0, x1


def key(seed: int) -> np.ndarray:
    """``jax.random.key(seed)`` data for a non-negative 32-bit seed."""
    return np.array([0, int(seed) & 0xFFFFFFFF], np.uint32)


def split(k, n: int = 2) -> np.ndarray:
    """``jax.random.split(k, n)`` -> ``(n, 2)`` uint32."""
    k = np.asarray(k, np.uint32)
    i = np.arange(n, dtype=np.uint32)
    a, b = threefry2x32(k[0], k[1], np.zeros_like(i), i)
    return np.stack([a, b], axis=-1)


def fold_in(k, data: int) -> np.ndarray:
    k = np.asarray(k, np.uint32)
    a, b = threefry2x32(k[0], k[1], np.uint32(0), np.uint32(data))
    return np.array([a, b], np.uint32)


def random_bits(k, n: int) -> np.ndarray:
    """32-bit ``random_bits`` of shape ``(n,)``."""
    k = np.asarray(k, np.uint32)
    i = np.arange(n, dtype=np.uint32)
    a, b = threefry2x32(k[0], k[1], np.zeros_like(i), i)
    return a ^ b


def uniform(k, n: int) -> np.ndarray:
    """``jax.random.uniform(k, (n,))`` float32 in [0, 1)."""
    bits = random_bits(k, n)
    f = ((bits >> np.uint32(9)) | np.uint32(0x3F800000)).view(np.float32)
    return (f - np.float32(1.0)).astype(np.float32)


def bernoulli(k, n: int, p: float = 0.5) -> np.ndarray:
    """``jax.random.bernoulli(k, p, (n,))``: ``uniform(k, (n,)) < p``."""
    return uniform(k, n) < np.float32(p)


def advance_iteration(k) -> np.ndarray:
    """The run key after one ns_step iteration (nested_sampling.py:465-466)."""
    return split(split(k, 2)[0], 5)[0]


def randint_array(k, n: int, lo: int, hi: int) -> np.ndarray:
    """``jax.random.randint(k, (n,), lo, hi)`` int32: with ``k1, k2 =
    split(k)``, element i combines ``higher = bits(k1)[i]`` and ``lower =
    bits(k2)[i]`` as ``((higher % span) * m + lower % span) % span`` in
    wrapping uint32 arithmetic, ``m = (2**16 % span)**2 % span``."""
    k1, k2 = split(k, 2)
    higher = random_bits(k1, n)
    lower = random_bits(k2, n)
    span = np.uint32(max(int(hi) - int(lo), 1))
    mult = np.uint32(65536 % int(span))
    mult = np.uint32((int(mult) * int(mult)) % int(span))
    with np.errstate(over="ignore"):
        off = ((higher % span) * mult + (lower % span)) % span
    return (np.int64(lo) + off.astype(np.int64)).astype(np.int32)
