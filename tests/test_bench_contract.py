"""The benchmark's reference arm runs on the host cores only: its JSON line must
carry the fields the benchmark contract names (metric, value, unit, impl, e2e with
zero transfer bytes, cpu_baseline with the core count).  Runs on CPU."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_json_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "3", "--cpu-seconds", "0.5"], capture_output=True, text=True, timeout=600,
                         cwd=ROOT, env={**os.environ, "CUDA_VISIBLE_DEVICES": ""})
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["metric"] == "scan positions/s per iteration" and line["unit"] == "positions/s"
    assert line["higher_is_better"] is True and line["value"] > 0
    assert line["steps"] == 1 and line["warmup"] == 3
    assert line["e2e"]["value"] == line["value"]
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    cb = line["cpu_baseline"]
    # without a GPU the sample's data cannot be simulated, so the arm reports the oracle port
    assert cb["kind"] == "port" and cb["reference_unavailable"]
    assert cb["cores"] >= 1 and cb["value"] == line["value"] and cb["sample"]
    assert "workload" in line["config"]
