"""The bench's multi-rank launch path on CPU: two gloo ranks under torchrun, reference arm.

Rank 0 alone times a full CPU-restatement solve of the (here 16-sphere) workload and prints one
JSON line; rank 1 exits without work.
"""
import json
import os
import subprocess
import sys

from conftest import ROOT


def test_reference_arm_under_two_gloo_ranks():
    env = dict(os.environ, OMP_NUM_THREADS="2")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr=127.0.0.1", "--master-port=29631", str(ROOT / "bench.py"), "--impl", "reference",
           "--gpus", "2", "--steps", "1", "--warmup", "0", "--spheres", "16"]
    out = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, out.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["cpu_baseline"]["kind"] == "port" and d["e2e"]["h2d_bytes_per_step"] == 0
    assert "no extrapolation" in d["cpu_baseline"]["sample"] and d["steps"] == 1
