"""bench.py --gpus N started without torchrun starts N ranks itself (one process per
GPU over torch.distributed), and rank 0 alone prints the JSON line with the whole-job
value.  Checked without a GPU through --cpu-check: gloo ranks, the CPU oracle as each
rank's step."""

import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("gpus", [1, 2])
def test_bench_starts_one_rank_per_gpu(gpus):
    env = {k: v for k, v in os.environ.items() if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK", "MASTER_ADDR", "MASTER_PORT")}
    out = subprocess.run(
        [sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", str(gpus), "--cpu-check", "--steps", "2", "--warmup", "1"],
        capture_output=True, text=True, timeout=240, env=env, cwd=ROOT,
    )
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, out.stdout
    rec = json.loads(lines[0])
    assert rec["n_gpus"] == gpus and rec["steps"] == 2 and rec["warmup"] == 1
    assert rec["value"] > 0 and rec["ms_per_step"] > 0
