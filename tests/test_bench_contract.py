"""bench.py's reference arm where the reference has no CPU code for the workload: one JSON line
with impl "reference", the workload's metric and the reason (runs on the CPU, no GPU needed)."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("workload", ["realtime", "denoise", "render", "media", "textures"])
def test_reference_arm_prints_one_line(workload):
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--workload", workload],
                         cwd=ROOT, capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["metric"] and d["unavailable"]


def test_reference_arm_of_the_served_stream_times_the_cpu_path_tracer():
    """--impl reference for the default workload (the served stream): the reference's trace_image on
    whole sampled jobs of the stream, one JSON line with its Mrays/s and how it was sampled."""
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "0"],
                         cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["steps"] == 1
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"]["h2d_bytes_per_step"] == 0
