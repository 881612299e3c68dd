"""The reference arm of bench.py (`--impl reference`) on the host: one JSON
line with the bench contract's keys, timed on the C++/OpenMP restatement
(the C1 workload, so that it runs in seconds); `steps` is the number of whole
steps actually timed (at least three, at most K)."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_one_contract_line():
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--workload", "C1",
                          "--steps", "2", "--warmup", "1", "--cpu-budget", "5"],
                         cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
              "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
              "impl", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["value"] > 0 and d["unit"] == "steps/s"
    assert 2 <= d["steps"] <= 2 and d["warmup"] == 1
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": "steps/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}


def test_reference_arm_batched_forms_say_unavailable():
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--workload", "C4"],
                         cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0
    d = json.loads([l for l in out.stdout.splitlines() if l.startswith("{")][0])
    assert d["impl"] == "reference" and "unavailable" in d
