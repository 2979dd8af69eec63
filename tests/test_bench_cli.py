"""The bench's reference arms on the CPU: each prints one JSON line with the fields of the
bench contract (a short layer prefix keeps the headline arm to seconds)."""

import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
KEYS = {"metric", "value", "unit", "impl", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
        "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"}


def _line(*args):
    r = subprocess.run([sys.executable, "bench.py", *args], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout[-2000:]
    return json.loads(lines[0])


def _check(d):
    assert KEYS <= set(d), KEYS - set(d)
    assert d["impl"] == "reference" and d["value"] > 0 and d["higher_is_better"] is True
    cb = d["cpu_baseline"]
    assert {"value", "unit", "cores", "kind", "sample"} <= set(cb) and cb["cores"] >= 1 and cb["kind"] == "port"
    assert d["e2e"]["value"] == d["value"] and d["e2e"]["h2d_bytes_per_step"] == 0
    assert d["e2e"]["d2h_bytes_per_step"] == 0 and "workload" in d["config"]


def test_reference_arm_line():
    d = _line("--impl", "reference", "--steps", "1", "--warmup", "0", "--layers", "2")
    _check(d)
    assert d["unit"] == d["metric"] == "term-gate updates/s"


def test_batched_reference_arm_line():
    d = _line("--workload", "batched_tfim", "--impl", "reference", "--steps", "1", "--warmup", "0")
    _check(d)
    assert d["config"]["instances"] == 256


def test_learned_reference_arm_is_unavailable():
    d = _line("--workload", "learned_kicked_ising", "--impl", "reference")
    assert d["impl"] == "reference" and "unavailable" in d
