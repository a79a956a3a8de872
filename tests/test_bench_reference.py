"""The bench's reference arm (`bench.py --impl reference`) on the CPU: one JSON line on rank 0 with the metric,
unit and workload of the CUDA arm, the timed sample described, and an end-to-end figure with no host-device
copies; the other ranks of a multi-process launch print nothing."""

import json
import os
import subprocess
import sys
from pathlib import Path

REPO = Path(__file__).resolve().parents[1]
if str(REPO) not in sys.path:
    sys.path.insert(0, str(REPO))


def run_bench(*args, env=None):
    return subprocess.run([sys.executable, str(REPO / "bench.py"), *args], cwd=REPO, capture_output=True, text=True,
                          env=env, timeout=300)


def test_the_reference_arm_prints_one_line_of_the_contract():
    result = run_bench("--impl", "reference", "--steps", "1", "--warmup", "0", "--cells", "32,48,32")
    assert result.returncode == 0, result.stderr
    lines = [line for line in result.stdout.splitlines() if line.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference"
    assert line["metric"] == line["unit"] == "Mcell-substeps/s"
    assert line["higher_is_better"] is True and line["value"] > 0
    assert line["steps"] == 1 and line["n_gpus"] == 1
    assert line["config"]["cells"] == [32, 48, 32]
    assert line["config"]["workload"].startswith("32x48x32 plain FP32 fluid step, 4 MG V-cycles")
    assert len(line["config"]["workload"]) <= 128
    import bench
    from plume_b200.recipe.derived import derive
    from plume_b200.workloads import plain_step_recipe

    # the CUDA arm prints the same config for the same workload
    assert line["config"] == bench.bench_config(derive(plain_step_recipe((32, 48, 32), cycles=4)), 4, 1)
    baseline = line["cpu_baseline"]
    assert baseline["kind"] == "port" and baseline["cores"] >= 1 and baseline["value"] == line["value"]
    assert "whole-grid substeps" in baseline["sample"]
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}


def test_only_rank_zero_runs_the_reference_arm():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    result = run_bench("--impl", "reference", "--steps", "1", "--warmup", "0", "--cells", "32,48,32", env=env)
    assert result.returncode == 0, result.stderr
    assert result.stdout.strip() == ""
