"""Helpers of the target-decoy statistics (reference ``vulcan/stats/_util.py``).

Same names and meaning as the reference: ``as_codes`` (dense int64 codes of any key array), ``segment_starts``,
``segment_cumsum`` / ``segment_reverse_cummin`` (running sum / reverse running minimum restarting at segment
starts), ``make_rng`` (seeded generator with sub-keys) and ``hash_tiebreak`` (storage-order-free tie-break keys:
splitmix64 of integer keys, ``_util.py:70-95``).
"""
from __future__ import annotations

import hashlib

import numpy as np

_U = np.uint64


def make_rng(seed=None, *keys) -> np.random.Generator:
    if isinstance(seed, np.random.Generator):
        return seed
    if seed is None:
        return np.random.default_rng()
    return np.random.default_rng(np.random.SeedSequence([int(seed)] + [int(k) for k in keys]))


def as_codes(x) -> np.ndarray:
    x = np.asarray(x)
    if x.ndim == 1 and x.dtype.kind in "iu":
        return x.astype(np.int64, copy=False)
    return np.unique(x, return_inverse=True)[1].astype(np.int64).ravel()


def segment_starts(sorted_keys: np.ndarray) -> np.ndarray:
    k = np.asarray(sorted_keys)
    m = np.ones(len(k), dtype=bool)
    if len(k) > 1:
        m[1:] = k[1:] != k[:-1]
    return m


def segment_cumsum(values: np.ndarray, starts: np.ndarray) -> np.ndarray:
    v = np.asarray(values)
    c = np.cumsum(v, dtype=np.int64 if v.dtype.kind in "biu" else np.float64)
    seg = np.cumsum(starts) - 1
    before = np.concatenate([np.zeros(1, c.dtype), c])[np.flatnonzero(starts)]
    return c - before[seg]


def segment_reverse_cummin(values: np.ndarray, starts: np.ndarray, cap: float = 1.0) -> np.ndarray:
    """Minimum over each element and everything after it in its segment, values clipped to [0, cap]."""
    v = np.minimum(np.asarray(values, np.float64), cap)
    seg = (np.cumsum(starts) - 1).astype(np.float64)
    shift = (2.0 * cap + 1.0) * seg      # later segments sit higher, so a running minimum never crosses back
    w = np.minimum.accumulate((v + shift)[::-1])[::-1]
    return w - shift


def _mix64(x: np.ndarray) -> np.ndarray:
    with np.errstate(over="ignore"):
        z = x.astype(_U) + _U(0x9E3779B97F4A7C15)
        z = (z ^ (z >> _U(30))) * _U(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> _U(27))) * _U(0x94D049BB133111EB)
        return z ^ (z >> _U(31))


def hash_tiebreak(keys, seed: int) -> np.ndarray:
    k = np.asarray(keys)
    if k.dtype.kind in "iu":
        return _mix64(k.astype(_U) ^ _mix64(np.array([seed], dtype=_U))[0])
    tag = str(int(seed)).encode()
    return np.fromiter((int.from_bytes(hashlib.blake2b(str(x).encode() + b"|" + tag, digest_size=8).digest(),
                                       "little") for x in k.ravel()), dtype=_U, count=k.size)
