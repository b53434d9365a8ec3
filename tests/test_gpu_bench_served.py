"""bench.py's served line: a short stream of small fits through dr_server_*, with the CPU baseline timed on one job's
image and the FP32 kernels' posterior-mean error against the FP64 oracle on that image (identical draws)."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.gpu
def test_served_line_carries_the_cpu_baseline_and_the_fp64_error():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--workload", "served_tiny", "--steps", "3",
                        "--warmup", "1", "--cpu-seconds", "1"], capture_output=True, text=True, timeout=900, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-3000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["metric"] == "served HMC gradient evals/sec" and line["value"] > 0
    assert line["latency_s"]["p99"] >= line["latency_s"]["p50"] > 0
    cb = line["cpu_baseline"]
    assert cb["kind"] == "port" and cb["value"] > 0 and cb["cores"] >= 1, cb
    assert "served job's image" in cb["sample"]
    pm = cb["posterior_mean_vs_fp64"]
    assert "error" not in pm, pm
    # FP32 kernels against the FP64 oracle on the same momentum draws and accept uniforms
    assert pm["rel_mean"] < 1e-3 and pm["accept_flips"] == 0, pm
