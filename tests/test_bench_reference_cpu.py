"""bench.py's reference arm runs on the host alone (the C restatement on every host thread)
and prints one JSON line: the same metric and config as the GPU arm, with
`impl`, `cpu_baseline` and a zero-copy `e2e`."""

import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_json_line():
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "0"],
                       cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["metric"] == "MPM particle-substeps/s" and line["unit"] == "particle-substeps/s"
    assert line["higher_is_better"] is True and line["value"] > 0
    assert line["config"]["workload"].startswith("mixed_500k")
    cb = line["cpu_baseline"]
    assert cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["sample"] and cb["value"] == line["value"]
    e = line["e2e"]
    assert e["value"] == line["value"] and e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0
