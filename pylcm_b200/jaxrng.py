"""A NumPy restatement of JAX's default random stream (64-bit mode).

The reference simulates with ``jax.random`` (``src/_lcm/simulation/random.py:
9-75``, ``simulate.py:465-668``, ``transitions.py:279-340``).  Its default
generator is the counter-based Threefry-2x32 hash with 20 rounds (Salmon,
Moraes, Dror and Shaw 2011, "Parallel random numbers: as easy as 1, 2, 3"),
driven by JAX's conventions, restated here:

- a key is a pair of uint32 words; ``key(seed)`` is (seed >> 32, seed & 0xffffffff);
- ``split(key, n)`` (the partitionable layout, JAX's default): key i is the
  hash of the counter pair (i >> 32, i & 0xffffffff) under `key`;
- 64 random bits of a key (one draw of shape ()): the hash of the counter
  pair (0, 0), high word first;
- ``uniform``: the 52 high bits as the mantissa of a float in [1, 2), minus
  one, scaled to [minval, maxval) and clamped below at minval;
- ``normal``: sqrt(2) erfinv(u) with u uniform on (nextafter(-1, 0), 1);
- ``choice(key, a, p=p)``: the first index whose cumulative weight reaches
  total * (1 - u);
- ``gumbel``: -log(-log(u)), u uniform on [tiny, 1);
- ``bernoulli(key, p)``: u < p.

Everything works on arrays of keys (shape (..., 2), uint32), one draw per key.
The normal sampler's inverse error function is the caller's (SciPy on the
host, CUDA's ``erfinv`` on the device); the uniform it transforms is exact.
"""

from __future__ import annotations

import numpy as np

_ROT = ((13, 15, 26, 6), (17, 29, 16, 24))
_PARITY = np.uint32(0x1BD11BDA)


def _rotl(x: np.ndarray, r: int) -> np.ndarray:
    return (x << np.uint32(r)) | (x >> np.uint32(32 - r))


def threefry2x32(k0, k1, x0, x1) -> tuple[np.ndarray, np.ndarray]:
    """Threefry-2x32 with 20 rounds of counters (x0, x1) under key (k0, k1)
    (uint32 arrays, broadcast against each other)."""
    k0, k1, x0, x1 = (np.asarray(v, dtype=np.uint32) for v in (k0, k1, x0, x1))
    k0, k1, x0, x1 = np.broadcast_arrays(k0, k1, x0, x1)
    ks = (k0, k1, k0 ^ k1 ^ _PARITY)
    with np.errstate(over="ignore"):
        x0 = x0 + ks[0]
        x1 = x1 + ks[1]
        for i in range(5):
            for r in _ROT[i % 2]:
                x0 = x0 + x1
                x1 = _rotl(x1, r)
                x1 = x1 ^ x0
            x0 = x0 + ks[(i + 1) % 3]
            x1 = x1 + ks[(i + 2) % 3] + np.uint32(i + 1)
    return x0, x1


def key(seed: int) -> np.ndarray:
    """``jax.random.key(seed)`` of a non-negative 64-bit seed: (hi, lo) words."""
    seed = int(seed) & 0xFFFFFFFFFFFFFFFF
    return np.array([seed >> 32, seed & 0xFFFFFFFF], dtype=np.uint32)


def split(keys, n: int) -> np.ndarray:
    """``jax.random.split(k, n)`` of every key in `keys` (shape (..., 2)):
    shape (..., n, 2)."""
    keys = np.asarray(keys, dtype=np.uint32)
    i = np.arange(n, dtype=np.uint64)
    hi = (i >> np.uint64(32)).astype(np.uint32)
    lo = (i & np.uint64(0xFFFFFFFF)).astype(np.uint32)
    k0 = keys[..., 0][..., None]
    k1 = keys[..., 1][..., None]
    b0, b1 = threefry2x32(k0, k1, hi, lo)
    return np.stack([b0, b1], axis=-1)


def bits64(keys) -> np.ndarray:
    """64 random bits per key (a draw of shape ())."""
    keys = np.asarray(keys, dtype=np.uint32)
    b0, b1 = threefry2x32(keys[..., 0], keys[..., 1], 0, 0)
    return (b0.astype(np.uint64) << np.uint64(32)) | b1.astype(np.uint64)


def uniform(keys, minval=0.0, maxval=1.0) -> np.ndarray:
    """One float64 in [minval, maxval) per key."""
    b = bits64(keys)
    f = ((b >> np.uint64(12)) | np.uint64(0x3FF0000000000000)).view(np.float64) - 1.0
    minval = np.asarray(minval, dtype=np.float64)
    maxval = np.asarray(maxval, dtype=np.float64)
    return np.maximum(minval, f * (maxval - minval) + minval)


def normal(keys, erfinv) -> np.ndarray:
    """One standard normal per key: sqrt(2) erfinv(u), u uniform on
    (nextafter(-1, 0), 1); `erfinv` is the inverse error function to use."""
    lo = np.nextafter(-1.0, 0.0)
    u = uniform(keys, lo, 1.0)
    return np.sqrt(2.0) * erfinv(u)


def uniform_shaped(keys, m: int, minval=0.0, maxval=1.0) -> np.ndarray:
    """``uniform(key, (m,))`` per key: element i from the counters (0, i);
    shape (..., m)."""
    keys = np.asarray(keys, dtype=np.uint32)
    i = np.arange(m, dtype=np.uint32)
    b0, b1 = threefry2x32(keys[..., 0][..., None], keys[..., 1][..., None], 0, i)
    b = (b0.astype(np.uint64) << np.uint64(32)) | b1.astype(np.uint64)
    f = ((b >> np.uint64(12)) | np.uint64(0x3FF0000000000000)).view(np.float64) - 1.0
    minval = np.asarray(minval, dtype=np.float64)
    maxval = np.asarray(maxval, dtype=np.float64)
    return np.maximum(minval, f * (maxval - minval) + minval)


def gumbel_shaped(keys, m: int) -> np.ndarray:
    """``jax.random.gumbel(key, (m,))`` per key: shape (..., m)."""
    u = uniform_shaped(keys, m, np.finfo(np.float64).tiny, 1.0)
    return -np.log(-np.log(u))


def gumbel(keys) -> np.ndarray:
    u = uniform(keys, np.finfo(np.float64).tiny, 1.0)
    return -np.log(-np.log(u))


def bernoulli(keys, p) -> np.ndarray:
    return uniform(keys) < np.asarray(p, dtype=np.float64)


def choice_index(keys, p) -> np.ndarray:
    """Index drawn by ``jax.random.choice(k, a, p=p)`` per key (rows of p):
    the first index whose cumulative weight reaches total * (1 - u)."""
    p = np.asarray(p, dtype=np.float64)
    cum = np.cumsum(p, axis=-1)
    r = cum[..., -1] * (1.0 - uniform(keys))
    return np.minimum((cum < r[..., None]).sum(axis=-1), p.shape[-1] - 1)


def simulation_keys(k: np.ndarray, names: list[str], n: int) -> tuple[np.ndarray, dict]:
    """``generate_simulation_keys`` (``random.py:9-75``): for each name in
    order, split the running key into n + 1 keys, keep the first as the
    running key and give the rest to the n subjects."""
    out = {}
    for name in names:
        ks = split(k, n + 1)
        k = ks[0]
        out[name] = ks[1:]
    return k, out
