"""bench.py's reference arm on the CPU: the JSON line the driver reads (impl,
metric, value, unit, cpu_baseline, e2e with no host<->device bytes), and the
torchrun rule that only rank 0 runs and prints it."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ARGS = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
        "--workload", "sinusoid256", "--steps", "2", "--warmup", "1", "--cpu-sample", "8"]


def _run(env_extra):
    env = dict(os.environ, **env_extra)
    return subprocess.run(ARGS, cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)


def test_reference_arm_line():
    p = _run({"RANK": "0", "WORLD_SIZE": "1"})
    assert p.returncode == 0, p.stderr[-2000:]
    line = json.loads(p.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["metric"] == "EMD signals/s (FP64)" and line["unit"] == "signals/s"
    assert line["value"] > 0 and line["higher_is_better"] is True
    assert line["steps"] == 2 and line["warmup"] == 1
    cb = line["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == line["value"]
    e2e = line["e2e"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0
    assert e2e["value"] == line["value"] and e2e["unit"] == line["unit"]
    assert line["config"]["workload"] == "sinusoid256"


def test_reference_arm_other_ranks_print_nothing():
    p = _run({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"})
    assert p.returncode == 0, p.stderr[-2000:]
    assert p.stdout.strip() == ""
