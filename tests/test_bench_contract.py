"""bench.py's reference arm (the CPU oracle timed on the host cores) keeps
the JSON-line contract on CPU: one line with the metric, value, unit, the
reference marker, a cpu_baseline describing the run and an e2e entry with no
host-device traffic; the batched workload, which the reference cannot run,
prints its `unavailable` line and exits 0."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(*args):
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args],
                         capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, out.stdout
    return json.loads(lines[0])


def test_reference_arm_line(oracle):
    d = _run("--impl", "reference", "--config", "n4096", "--steps", "1", "--warmup", "3")
    assert d["impl"] == "reference"
    import bench
    assert d["metric"] == bench.METRIC and d["unit"] == "solves/s"
    assert d["higher_is_better"] is True and d["steps"] == 1 and d["warmup"] == 3
    assert d["value"] > 0 and d["ms_per_step"] > 0
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": "solves/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}
    assert d["config"]["relres"] < 1e-12       # the oracle solved the system


def test_batched_workload_reference_unavailable():
    d = _run("--impl", "reference", "--config", "batch64")
    assert d["impl"] == "reference" and "unavailable" in d
