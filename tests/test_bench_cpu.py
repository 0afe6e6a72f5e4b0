"""bench.py on the CPU: the reference arm prints one JSON line of the bench
contract (rank 0 only), and the product arm fails loudly without a GPU (there
is no CPU fallback to time)."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BENCH = os.path.join(ROOT, "bench.py")


def run_bench(args, env_extra=None, timeout=600):
    env = dict(os.environ)
    env.update(env_extra or {})
    return subprocess.run([sys.executable, BENCH] + args, capture_output=True, text=True, timeout=timeout,
                          cwd=ROOT, env=env)


def test_reference_arm_prints_the_contract_line():
    res = run_bench(["--impl", "reference", "--steps", "1", "--warmup", "1"])
    assert res.returncode == 0, res.stderr[-2000:]
    lines = [l for l in res.stdout.splitlines() if l.strip().startswith("{")]
    assert len(lines) == 1, res.stdout
    line = json.loads(lines[0])
    assert line["impl"] == "reference"
    assert line["metric"] == "spectral paths/s" and line["unit"] == "spectral paths/s"
    assert line["value"] > 0 and line["higher_is_better"] is True
    assert line["steps"] == 1 and line["warmup"] == 1 and line["n_gpus"] == 1
    assert line["config"]["workload"] == "heavy-geometry-1.0M-tri-dome"
    assert line["config"]["triangles"] == 1000480
    base = line["cpu_baseline"]
    assert base["kind"] in ("reference", "port") and base["cores"] >= 1 and base["value"] == line["value"]
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}


def test_reference_arm_runs_on_rank_zero_only():
    res = run_bench(["--impl", "reference", "--steps", "1", "--warmup", "1"],
                    env_extra={"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"})
    assert res.returncode == 0, res.stderr[-2000:]
    assert not [l for l in res.stdout.splitlines() if l.strip().startswith("{")]


def test_product_arm_fails_loudly_without_a_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    res = run_bench(["--steps", "1", "--warmup", "0", "--no-autotune", "--no-cpu-baseline"], timeout=300)
    assert res.returncode != 0
    assert not [l for l in res.stdout.splitlines() if l.strip().startswith('{"metric"')]
