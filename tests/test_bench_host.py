"""bench.py's reference arm (--impl reference: the FP64 CPU restatement on the host cores)
through its command line, CPU only: the JSON line's keys, and the workload it reports is
the one our arm reports for the same number of GPUs (single-GPU run, or the weak-scaled
decomposition as rank 0 of a torchrun launch; other ranks print nothing)."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def reference_line(extra_env):
    env = dict(os.environ, PIP_REF_BUDGET_S="1", **extra_env)
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--steps", "1", "--warmup", "1"], cwd=ROOT, env=env,
                         capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    return json.loads(lines[-1]) if lines else None


def test_reference_arm_single_gpu():
    d = reference_line({})
    for k in ("metric", "value", "unit", "impl", "n_gpus", "steps", "warmup", "ms_per_step",
              "higher_is_better", "scaling", "dtype", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] == "port"
    assert "1024x1024" in d["config"]["workload"] and d["config"]["cells"] == 1024 * 1024


@pytest.mark.parametrize("rank", [0, 1])
def test_reference_arm_under_torchrun(rank):
    d = reference_line({"WORLD_SIZE": "2", "RANK": str(rank), "LOCAL_RANK": str(rank)})
    if rank == 1:
        assert d is None
        return
    assert "y-slab" in d["config"]["workload"] and d["config"]["cells"] == 2 * 1024 * 1024
