"""bench.py's reference arm (the CPU restatement timed on the host cores) at
a small size: one JSON line with the fields the benchmark contract asks for,
on the same metric as the B200 arm."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_json_line(oracle_lib):
    out = subprocess.run(
        [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
         "--nvis", "4000", "--grid", "256", "--oversampling", "8",
         "--steps", "1", "--warmup", "1"],
        capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    sys.path.insert(0, ROOT)
    import bench
    assert line["impl"] == "reference"
    assert line["metric"] == bench.METRIC and line["unit"] == bench.UNIT
    assert line["value"] > 0 and line["higher_is_better"] is True
    assert line["steps"] == 1 and line["warmup"] == 1
    assert line["config"]["workload"].startswith(
        "full-pol degrid+grid 256x256x4") and "os 8" in line["config"]["workload"]
    cb = line["cpu_baseline"]
    assert cb["value"] == line["value"] and cb["kind"] == "port"
    assert cb["cores"] >= 1
    e2e = line["e2e"]
    assert e2e["value"] == line["value"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0
