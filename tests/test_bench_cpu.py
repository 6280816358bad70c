"""bench.py's reference arm on the CPU: one JSON line on stdout with the contract's keys
(the reference's own progress output stays off stdout), and ranks other than 0 print
nothing.  The workload is the small Q4 64x64 case so that the test takes seconds."""
import json
import os
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def _run(extra_env=None):
    env = dict(os.environ)
    env.update(extra_env or {})
    cmd = [sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--config", "q4_64",
           "--steps", "1", "--warmup", "1"]
    return subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)


def test_reference_arm_prints_one_json_line():
    res = _run()
    assert res.returncode == 0, res.stderr[-2000:]
    lines = [ln for ln in res.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1, res.stdout[-2000:]
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
                "higher_is_better", "config", "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["value"] > 0 and d["e2e"]["value"] == d["value"]
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    assert d["cpu_baseline"]["kind"] in ("reference", "port")
    assert d["cpu_baseline"]["cores"] >= 1 and d["config"]["workload"] == "q4_64"
    # same steps and warm-up as the GPU arm (which takes at least 3 warm-up steps), and
    # the full workload mesh in the same config object the GPU arm prints
    assert d["steps"] == 1 and d["warmup"] == 3
    assert d["config"]["elements"] == 64 * 64 and d["config"]["dofs"] == 65 * 65 * 2
    sys.path.insert(0, str(ROOT))
    import bench
    from gpufem_b200 import meshgen as mg
    assert d["config"] == bench.workload_config("q4_64", mg.workload("q4_64"), 1)


def test_reference_arm_other_ranks_print_nothing():
    res = _run({"RANK": "1", "LOCAL_RANK": "1", "WORLD_SIZE": "2"})
    assert res.returncode == 0, res.stderr[-2000:]
    assert res.stdout.strip() == ""
