"""bench.py's reference arm where the reference has no CPU code for the workload: one JSON line
with impl "reference", the workload's metric and the reason (runs on the CPU, no GPU needed)."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("workload", ["realtime", "denoise", "serve", "render", "media", "textures"])
def test_reference_arm_prints_one_line(workload):
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--workload", workload],
                         cwd=ROOT, capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["metric"] and d["unavailable"]
