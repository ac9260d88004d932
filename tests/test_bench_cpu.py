"""bench.py's reference arm: the reference's own test_ycsb (oracle/_ref) on
the workload's shape when it can run, and the project's CPU port of the CC
rules beside it. On a machine without a GPU the reference cannot run, so the
line says so (`unavailable`) and still carries the CPU port's measurement;
with a GPU it keeps the bench contract's keys. Small case."""
import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def test_reference_arm_line():
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference",
                          "--rows", "65536", "--txs", "16384", "--steps", "1", "--warmup", "1",
                          "--cpu-threads", "2"],
                         capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert out.returncode == 0, out.stderr
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    port = line["cpu_port"]
    assert port["cores"] == 2 and port["kind"] == "port" and port["value"] > 0
    if "unavailable" in line:
        assert line["unavailable"]
        return
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
              "higher_is_better", "scaling", "vs_baseline", "dtype", "config", "cpu_baseline",
              "e2e"):
        assert k in line, k
    assert line["value"] > 0 and line["cpu_baseline"]["kind"] == "reference"
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["value"] == line["value"]
