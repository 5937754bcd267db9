"""Seeded synthetic job streams for batched and served proving.

* `shape_for_mu`: the reference-valid matrix shape of a 2^mu polynomial, log_m = min(7,
  floor((mu - 7) / 2)), inside setup's shared-domain window (pcs/src/ligesis.rs:246-251).
* `batch_mus`: 96 sizes mu = floor(14 + 8u), u uniform from seed 5 (log-uniform sizes in
  [2^14, 2^22)).
* `serve_stream`: Poisson arrivals (exponential gaps, default mean 5 ms = 200 jobs/s), mu =
  floor(14 + 11u) clipped to 24, and a `gpt2_fraction` of requests replaced by the merged
  integer GPT-2 layer witness of `gpt2_layer_witness`.
* `gpt2_layer_witness`: int8-range weights 768 x 768 and activations 64 x 768 from seed 6,
  lifted to Goldilocks like proofsys' `encode_i64` (negative x -> p - |x|,
  proofsys/src/witness.rs:102-108), each padded to 1024 columns and to a power-of-two row count
  (proofsys/src/canonical.rs:119-127) and stacked with the instance index on the high variables
  (proofsys/src/commit.rs:32-41): two instances of 2^20 elements, mu = 21.
"""
from __future__ import annotations

import math

import numpy as np

from . import rng

P = rng.P


def shape_for_mu(mu: int) -> tuple[int, int]:
    log_m = min(7, (mu - 7) // 2)
    return log_m, mu - log_m


def _uniform01(seed: int, count: int, start: int = 0) -> np.ndarray:
    return (rng.words(seed, start, count) >> np.uint64(11)).astype(np.float64) / float(1 << 53)


def batch_mus(n: int = 96, seed: int = 5, lo: int = 14, span: int = 8) -> list[int]:
    return [int(lo + span * u) for u in _uniform01(seed, n)]


def encode_i64(x: np.ndarray) -> np.ndarray:
    x = np.asarray(x, dtype=np.int64)
    out = x.astype(np.uint64)
    neg = x < 0
    out[neg] = np.uint64(P) - (-x[neg]).astype(np.uint64)
    return out


def gpt2_layer_witness(seed: int = 6) -> np.ndarray:
    w = (rng.words(seed, 0, 768 * 768) % np.uint64(256)).astype(np.int64) - 128
    a = (rng.words(seed, 768 * 768, 64 * 768) % np.uint64(256)).astype(np.int64) - 128
    elem = 1 << 20
    out = np.zeros(2 * elem, dtype=np.uint64)
    wm = np.zeros((1024, 1024), dtype=np.uint64)
    wm[:768, :768] = encode_i64(w).reshape(768, 768)
    am = np.zeros((64, 1024), dtype=np.uint64)
    am[:, :768] = encode_i64(a).reshape(64, 768)
    out[:elem] = wm.reshape(-1)
    out[elem:elem + am.size] = am.reshape(-1)
    return out


def serve_stream(n: int, rate_per_s: float = 200.0, seed: int = 7, lo: int = 14, hi: int = 24,
                 gpt2_fraction: float = 0.1):
    """[(arrival_s, mu, kind)] with kind 'poly' or 'gpt2'."""
    u_gap = _uniform01(seed, n)
    u_mu = _uniform01(seed + 1, n)
    u_kind = _uniform01(seed + 2, n)
    t = 0.0
    out = []
    for i in range(n):
        t += -math.log(1.0 - u_gap[i]) / rate_per_s
        if u_kind[i] < gpt2_fraction:
            out.append((t, 21, "gpt2"))
        else:
            out.append((t, min(hi, int(lo + (hi - lo + 1) * u_mu[i])), "poly"))
    return out
