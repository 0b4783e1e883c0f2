"""bench.py's output contract on CPU: the committed traffic table, the
measured peak, and the reference arm's JSON line on a small mesh."""
from __future__ import annotations

import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_traffic_table_has_every_default_line():
    sys.path.insert(0, ROOT)
    import bench
    for prec in ("fp64", "mixed"):
        for path in ("tiles", "node-tiles"):
            v = bench.profiled_traffic("disk1p8m", prec, path)
            assert v is not None and 3e8 < v < 2e9, (prec, path, v)
    # The one-kernel step moves fewer bytes than the two-kernel step.
    assert bench.profiled_traffic("disk1p8m", "fp64", "node-tiles") < bench.profiled_traffic("disk1p8m", "fp64", "tiles")
    assert bench.profiled_traffic("disk1p8m", "fp64", "cluster") is None


def test_measured_peak_read_from_file():
    sys.path.insert(0, ROOT)
    import bench
    peak, kind = bench.measured_peak_hbm()
    if os.path.exists(os.path.join(ROOT, "MEASURED_PEAKS.json")):
        assert kind == "measured" and 3000 < peak < 9000
    else:
        assert kind == "fallback"


def test_reference_arm_json_line():
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--workload", "disk50", "--steps", "3",
                          "--warmup", "3"], cwd=ROOT, capture_output=True, text=True, timeout=600, env=env)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in line, k
    assert line["impl"] == "reference" and line["value"] > 0 and line["e2e"]["h2d_bytes_per_step"] == 0
    assert line["cpu_baseline"]["kind"] in ("reference", "port") and line["cpu_baseline"]["cores"] >= 1
    assert "spacing 0.05" in line["config"]["workload"]


def test_reference_arm_under_torchrun_prints_one_line():
    """Launched as the multi-GPU bench is (torchrun, two ranks), the reference
    arm runs on rank 0 alone and prints exactly one JSON line."""
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr",
           "127.0.0.1", "--master-port", str(port), "bench.py", "--impl", "reference", "--gpus", "2",
           "--workload", "disk50", "--steps", "3", "--warmup", "3"]
    out = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600, env=env)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
