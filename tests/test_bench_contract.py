"""The reference arm of bench.py on the CPU: `--impl reference` times the FP64 oracle port of the
reference's algorithm on the host cores and prints one JSON line with the benchmark's metric,
config and the e2e / cpu_baseline objects; under torchrun only rank 0 prints."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(env_extra, tmp_path):
    env = dict(os.environ, **env_extra)
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--W", "160",
                           "--H", "120", "--steps", "3", "--warmup", "3"], cwd=str(tmp_path), env=env,
                          capture_output=True, text=True, timeout=300)


def test_reference_arm_prints_one_line(tmp_path):
    p = _run({}, tmp_path)
    assert p.returncode == 0, p.stderr
    lines = [ln for ln in p.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["metric"] == "cell-updates/s" and d["unit"] == "cell-updates/s"
    assert d["higher_is_better"] is True and d["steps"] == 3 and d["warmup"] == 3 and d["value"] > 0
    assert d["config"]["grid_cells"] == 160 * 120 and "workload" in d["config"]
    cpu = d["cpu_baseline"]
    assert cpu["kind"] == "port" and cpu["cores"] >= 1 and cpu["value"] == d["value"] and cpu["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_do_no_work(tmp_path):
    p = _run({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"}, tmp_path)
    assert p.returncode == 0, p.stderr
    assert p.stdout.strip() == ""
