"""The benchmark's JSON line, checked on the CPU through its reference arm
(the CPU implementation of the path timed on the host cores): one line with
the keys the benchmark contract requires, `cpu_baseline` and `e2e` objects
describing that run, and a positive time."""
import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]

REQUIRED = ["metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
            "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config"]


def test_reference_arm_prints_the_contract_line():
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1",
                        "--warmup", "1"], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    for k in REQUIRED:
        assert k in d, k
    assert d["impl"] == "reference"
    assert d["value"] > 0 and d["ms_per_step"] == d["value"]
    assert d["higher_is_better"] is False and d["n_gpus"] == 1
    assert d["steps"] == 1 and d["warmup"] == 1
    assert isinstance(d["config"], dict) and "workload" in d["config"]
    # the same config object as the B200 arm's line (same workload, same keys)
    sys.path.insert(0, str(ROOT))
    import bench
    assert d["config"] == bench.CONFIG
    assert d["metric"] == bench.METRIC
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["unit"] == d["unit"]
    assert cb["kind"] in ("reference", "port") and cb["cores"] >= 1 and cb["sample"]
    e2e = d["e2e"]
    assert e2e["value"] == d["value"] and e2e["unit"] == d["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0
