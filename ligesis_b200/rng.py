"""Seeded, documented input generator (the reference draws from `rand::rng()`, which is not
reproducible; this build fixes explicit inputs instead, and both the GPU prover and the CPU
oracle consume the identical buffers).

Counter-based SplitMix64: word(seed, i, t) = mix64(seed * 0x9E3779B97F4A7C15
+ (i + 1) * 0xD1B54A32D192ED03 + t * 0x8CB92BA72F3D8DD7)  (all mod 2^64), where mix64 is the
SplitMix64 finalizer.  A Goldilocks element i is the first word(seed, i, t), t = 0, 1, ...,
that is below p (rejection sampling, as `StandardUniform` for Goldilocks does); an EF element
i is the pair of Goldilocks elements 2i, 2i + 1; a raw u64 ("int") is word(seed, i, 0).
Every element depends only on (seed, i), so generation is vectorised.
"""
from __future__ import annotations

import numpy as np

P = 0xFFFFFFFF00000001
_K1 = np.uint64(0x9E3779B97F4A7C15)
_K2 = np.uint64(0xD1B54A32D192ED03)
_K3 = np.uint64(0x8CB92BA72F3D8DD7)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def _mix64(x: np.ndarray) -> np.ndarray:
    x = x ^ (x >> np.uint64(30))
    x = x * _M1
    x = x ^ (x >> np.uint64(27))
    x = x * _M2
    return x ^ (x >> np.uint64(31))


def words(seed: int, start: int, count: int, attempt: int = 0) -> np.ndarray:
    """Raw 64-bit words for indices [start, start + count)."""
    with np.errstate(over="ignore"):
        idx = np.arange(start, start + count, dtype=np.uint64)
        base = np.uint64(seed & 0xFFFFFFFFFFFFFFFF) * _K1 + np.uint64(attempt) * _K3
        return _mix64(base + (idx + np.uint64(1)) * _K2)


def field_elements(seed: int, count: int, start: int = 0) -> np.ndarray:
    """`count` uniform Goldilocks elements (canonical u64)."""
    out = words(seed, start, count, 0)
    bad = np.nonzero(out >= np.uint64(P))[0]
    attempt = 1
    while bad.size:
        with np.errstate(over="ignore"):
            idx = bad.astype(np.uint64) + np.uint64(start)
            base = np.uint64(seed & 0xFFFFFFFFFFFFFFFF) * _K1 + np.uint64(attempt) * _K3
            cand = _mix64(base + (idx + np.uint64(1)) * _K2)
        out[bad] = cand
        bad = bad[cand >= np.uint64(P)]
        attempt += 1
    return out


def ext_elements(seed: int, count: int, start: int = 0) -> np.ndarray:
    """`count` uniform EF elements as a (count, 2) u64 array of (c0, c1)."""
    return field_elements(seed, 2 * count, 2 * start).reshape(count, 2)


def ints(seed: int, count: int, start: int = 0) -> np.ndarray:
    """`count` raw u64 draws (the oracle's `next_int` values)."""
    return words(seed, start, count, 0)


class SeededRng:
    """Stand-in for the reference's `&mut impl Rng`: successive draws advance a counter, so a
    sequence of `setup`/`random_*` calls on one SeededRng is reproducible from its seed."""

    def __init__(self, seed: int):
        self.seed = int(seed)
        self.pos = 0

    def field_elements(self, count: int) -> np.ndarray:
        out = field_elements(self.seed, count, self.pos)
        self.pos += count
        return out

    def ext_elements(self, count: int) -> np.ndarray:
        out = field_elements(self.seed, 2 * count, self.pos).reshape(count, 2)
        self.pos += 2 * count
        return out

    def ints(self, count: int) -> np.ndarray:
        out = ints(self.seed, count, self.pos)
        self.pos += count
        return out
