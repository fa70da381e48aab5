"""bench.py's reference arm on the CPU: the JSON line it prints for a tiny
workload carries the keys the bench contract asks of it (the reference's own
mrrr() timed on the host cores, its results checked, e2e with no copies), or
an `unavailable` line when the reference library is not built."""
import json
import os
import subprocess
import sys

import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_json_line():
    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--count", "16",
           "--nmax", "128", "--steps", "1", "--warmup", "1", "--ref-step-seconds", "0.5"]
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    if oracle.ref_lib() is None:
        assert "unavailable" in line
        return
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
                "higher_is_better", "dtype", "config", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["value"] > 0 and line["higher_is_better"] is True
    assert line["steps"] == 1 and line["warmup"] == 1
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    assert line["e2e"]["value"] == line["value"]
    cb = line["cpu_baseline"]
    assert cb["kind"] in ("reference", "port") and cb["cores"] >= 1
    assert cb["checked"] is True and cb["checked_problems"] > 0
    assert "16 tridiagonals" in line["config"]["workload"]
