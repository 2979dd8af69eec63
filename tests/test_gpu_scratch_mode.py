"""The other modes of k_run_groups against the oracle.  Scratch mode (group outputs placed by
k_run_place, for sums with many groups) is taken from 2^18 groups on; with
PPVM_RUN_SCRATCH_MIN_GROUPS=1 every fused run with a group takes it.  Tiled mode (one
look-back per tile of groups), one group per warp and one group per lane are the three group
modes; by default a run of many single-member groups takes lane mode and the others one group
per warp, and PPVM_RUN_GROUP_MODE=tiled|warp|lanes forces one.  Both settings are read once
per process, so the fused-run parity tests run again in a child
process with each set: the term lists must match the oracle's bit for bit."""

import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_fused_runs_in_scratch_mode_match_the_oracle():
    env = dict(os.environ, PPVM_RUN_SCRATCH_MIN_GROUPS="1")
    r = subprocess.run([sys.executable, "-m", "pytest", "tests/test_gpu_parity.py", "-m", "gpu", "-x", "-q",
                        "-k", "fused or random or kicked or wide or growth or cached or reused"],
                       cwd=ROOT, env=env, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-2000:]
    assert " passed" in r.stdout


def test_fused_runs_in_tiled_mode_match_the_oracle():
    env = dict(os.environ, PPVM_RUN_GROUP_MODE="tiled")
    r = subprocess.run([sys.executable, "-m", "pytest", "tests/test_gpu_parity.py", "-m", "gpu", "-x", "-q",
                        "-k", "fused or random or kicked or wide or growth or cached or reused"],
                       cwd=ROOT, env=env, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-2000:]
    assert " passed" in r.stdout


def test_fused_runs_with_one_lookback_per_group_match_the_oracle():
    env = dict(os.environ, PPVM_RUN_GROUP_MODE="warp")
    r = subprocess.run([sys.executable, "-m", "pytest", "tests/test_gpu_parity.py", "-m", "gpu", "-x", "-q",
                        "-k", "fused or random or kicked or wide or growth or cached or reused or clifford_t"],
                       cwd=ROOT, env=env, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-2000:]
    assert " passed" in r.stdout


def test_fused_runs_in_lane_mode_match_the_oracle():
    env = dict(os.environ, PPVM_RUN_GROUP_MODE="lanes")
    r = subprocess.run([sys.executable, "-m", "pytest", "tests/test_gpu_parity.py", "-m", "gpu", "-x", "-q",
                        "-k", "fused or random or kicked or wide or growth or cached or reused or clifford_t"],
                       cwd=ROOT, env=env, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-2000:]
    assert " passed" in r.stdout
