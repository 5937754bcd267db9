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


def tiny_gpt():
    """The reference's own tiny model (proofsys/src/canonical.rs:318-361): one block, two
    positions, d_model 2, MLP 3, vocabulary 4, scale 4, max_v 2."""
    cfg = {"n_seq": 2, "d_model": 2, "mlp_hidden": 3, "vocab": 4, "scale": 4, "max_v": 2,
           "n_head": 1}
    a = lambda *v: np.array(v, dtype=np.int64)
    exp_lut = np.array([0 if i == 0 else 1 for i in range(2 * 4 + 1)], dtype=np.int64)
    gelu_lut = np.arange(2 * 2 * 4 + 1, dtype=np.int64) - 8
    w = {"ln_1_g": a(4, 4), "ln_1_b": a(0, 0),
         "attn_w": a(1, 0, 0, 1, 1, 0, 0, 1, 1, 0, 0, 1).reshape(2, 6), "attn_b": np.zeros(6, np.int64),
         "attn_proj_w": a(1, 0, 0, 1).reshape(2, 2), "attn_proj_b": a(0, 0),
         "ln_2_g": a(4, 4), "ln_2_b": a(0, 0), "fc_w": a(1, 0, 1, 0, 1, -1).reshape(2, 3),
         "fc_b": a(0, 0, 0), "fproj_w": a(1, 0, 0, 1, 1, -1).reshape(3, 2), "fproj_b": a(0, 0)}
    wte = a(1, 0, 0, 1, 1, 1, -1, 2).reshape(4, 2)
    x0 = a(1, -2, 3, 1).reshape(2, 2)
    return cfg, x0, w, a(4, 4), a(0, 0), wte, exp_lut, gelu_lut
