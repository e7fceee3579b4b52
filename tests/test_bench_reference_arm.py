"""bench.py --impl reference on the host: the JSON line of the reference arm (the C++ FP64
restatement of the reference on the host cores, no GPU needed)."""
from __future__ import annotations

import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def test_reference_arm_line():
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference",
                          "--workload", "sweep", "--points", "16", "--steps", "1",
                          "--warmup", "3"],
                         check=True, capture_output=True, text=True, timeout=600).stdout
    line = json.loads(out.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
              "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
              "cpu_baseline", "e2e"):
        assert k in line, k
    assert line["value"] > 0 and line["unit"] == "points/s" and line["higher_is_better"]
    assert line["warmup"] >= 3 and line["steps"] == 1
    assert line["config"]["workload"].startswith("sweep:")
    cb = line["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == line["value"]
    e2e = line["e2e"]
    assert e2e["value"] == line["value"] and e2e["h2d_bytes_per_step"] == 0
    assert "reference_js" in line["node_probe"]
