"""Shared test inputs: every buffer comes from ligesis_b200.rng, so the GPU path and the
oracle consume identical data."""
from __future__ import annotations

import numpy as np

from ligesis_b200 import rng

P = rng.P


def ligesis_inputs(log_m: int, log_n: int, seed: int = 1, oracle_len: int = 4096):
    """f (seed), A (seed+1), z (seed+2), oracle fields/ints (seed+3) for one shape."""
    mu = log_m + log_n
    f = rng.field_elements(seed, 1 << mu)
    A = rng.field_elements(seed + 1, 32 * (64 << log_m)).reshape(32, 64 << log_m)
    z = rng.ext_elements(seed + 2, mu)
    g = rng.SeededRng(seed + 3)
    fields = g.ext_elements(oracle_len)
    ints = g.ints(oracle_len)
    return f, A, z, fields, ints


def ef_list(a) -> list[tuple[int, int]]:
    a = np.asarray(a, dtype=np.uint64).reshape(-1, 2)
    return [(int(x), int(y)) for x, y in a]
