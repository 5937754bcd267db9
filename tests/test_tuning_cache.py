"""The committed launch-choice cache (ligesis_b200/tuning.json), which bench.py and ProverEngine
apply when they start: every entry holds only settings lgs_tune accepts (hash_ctas <= 4096,
sumcheck_blocks <= 296, hash_groups <= 8 row blocks), each kept setting is one the autotuner
actually timed, and it is no slower than the defaults in the same run.  Runs on the CPU (the
cache is read as a file, no device is asked for its name)."""
from __future__ import annotations

import pytest

from ligesis_b200 import autotune

LIMITS = {"hash_ctas": 4096, "sumcheck_blocks": 296, "hash_groups": 8}


def _entries():
    cache = autotune.load()
    assert cache, "the tuning cache is missing or empty"
    for gpu, shapes in cache.items():
        for key, entry in shapes.items():
            yield gpu, key, entry


@pytest.mark.parametrize("gpu,key,entry", list(_entries()),
                         ids=lambda v: v if isinstance(v, str) else "")
def test_cached_settings_are_valid_and_timed(gpu, key, entry):
    if key.startswith("engine"):
        assert int(key[len("engine"):]) > 0
        params = ("hash_ctas", "sumcheck_blocks")
        assert entry["pps"] >= entry["default_pps"]
        timed = [(t["hash_ctas"], t["sumcheck_blocks"]) for t in entry["trials"]]
        assert (entry["hash_ctas"], entry["sumcheck_blocks"]) in timed
        best = max(entry["trials"], key=lambda t: t["pps"])
        assert best["pps"] == entry["pps"]
    else:
        log_m, log_n = (int(v) for v in key.split("x"))
        assert autotune.shape_key(log_m, log_n) == key
        params = autotune.PARAMS
        assert entry["ms"] <= entry["default_ms"]
        timed = [(t["hash_ctas"], t["sumcheck_blocks"]) for t in entry["trials"]]
        assert (entry["hash_ctas"], entry["sumcheck_blocks"]) in timed
        groups = [t["hash_groups"] for t in entry["e2e_trials"]]
        assert entry["hash_groups"] in groups
        assert entry["e2e_ms"] == min(t["ms"] for t in entry["e2e_trials"])
    for p in params:
        assert isinstance(entry[p], int) and 0 <= entry[p] <= LIMITS[p], (gpu, key, p)


def test_bench_shape_is_cached_for_b200():
    """bench.py's line applies the entry for its own shape (2^7 x 2^17) on B200."""
    shapes = autotune.load().get("NVIDIA B200", {})
    assert "7x17" in shapes and autotune.engine_key(12) in shapes
