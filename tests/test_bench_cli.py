"""The bench's reference arms on the CPU: each prints one JSON line with the fields of the
bench contract, and the same ``config`` the GPU arm prints for that workload (a 2-layer
kicked-Ising circuit keeps the headline arm to seconds here)."""

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


def _gpu_arm_config(workload, layers=20):
    sys.path.insert(0, ROOT)
    import bench

    return bench.config_dict(bench.workload(workload, layers), 1)


def test_reference_arm_line():
    d = _line("--impl", "reference", "--steps", "1", "--warmup", "1", "--layers", "2")
    _check(d)
    assert d["unit"] == d["metric"] == "term-gate updates/s"
    assert d["config"] == _gpu_arm_config("kicked_ising_2d", 2)
    assert d["config"]["layers"] == 2 and d["config"]["gates_per_step"] == 2 * (264 + 144)
    assert d["result"]["term_gate_updates_per_step"] > 0


def test_tfim_reference_arm_line():
    d = _line("--workload", "tfim_1d", "--impl", "reference", "--steps", "2", "--warmup", "1")
    _check(d)
    assert d["config"] == _gpu_arm_config("tfim_1d")
    assert d["result"]["term_gate_updates_per_step"] == 64033


def test_clifford_t_workload_is_a_prefix_of_the_1000_layer_circuit():
    sys.path.insert(0, ROOT)
    import bench
    from ppvm_b200 import circuits as C

    wl = bench.workload("clifford_t")
    full = C.clifford_t(n=64, layers=1000, seed=0, p_t=0.05, thr=1e-6)
    assert wl.observable == full.observable and wl.ops == full.ops[:len(wl.ops)]
    assert bench.config_dict(wl, 1)["layers"] == 26


def test_batched_reference_arm_line():
    d = _line("--workload", "batched_tfim", "--impl", "reference", "--steps", "1", "--warmup", "0")
    _check(d)
    assert d["config"]["instances"] == 256


def test_learned_reference_arm_is_unavailable():
    d = _line("--workload", "learned_kicked_ising", "--impl", "reference")
    assert d["impl"] == "reference" and "unavailable" in d
