"""bench.py's reference arm runs on the host alone (the CPU restatement of the reference prover on
the line's workload), so its JSON line can be checked here at a small reference-valid shape
(2^3 x 2^10, selected with --log-m/--log-n as for the mu = 26 line): one line, the keys the line
contract asks for, the metric and config of that shape, commit and prove timed separately, and an
e2e entry with no host-device bytes."""
from __future__ import annotations

import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def test_reference_arm_prints_one_contract_line():
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference",
                          "--steps", "2", "--warmup", "0", "--log-m", "3", "--log-n", "10"], capture_output=True, text=True,
                         check=True, cwd=ROOT, timeout=600).stdout
    lines = [ln for ln in out.splitlines() if ln.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
                "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
                "impl", "cpu_baseline", "e2e"):
        assert key in d, key
    import bench

    assert d["impl"] == "reference" and d["unit"] == "ms"
    assert d["metric"] == bench.metric_for(3, 10) == "LigeSIS commit+eval ms at mu=13 (2^3 x 2^10)"
    assert bench.METRIC == bench.metric_for(7, 17)
    assert d["higher_is_better"] is False and d["value"] > 0
    assert d["steps"] == 2 and d["warmup"] == 3  # the harness raises warm-up to at least 3
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert d["cpu_baseline"]["value"] == d["value"]
    assert abs(d["stages_ms"]["commit"] + d["stages_ms"]["prove"] - d["value"]) < 0.2
    assert d["e2e"] == {"value": d["value"], "unit": "ms", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}
    assert d["config"]["workload"].startswith("LigeSIS commit+eval, mu=13 as 2^3 x 2^10")
    assert (d["config"]["log_m"], d["config"]["log_n"]) == (3, 10)
