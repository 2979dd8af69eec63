"""Scratch mode of the fused runs (group outputs placed by k_run_place, for sums with many
groups) against the oracle.  The library takes scratch mode from 2^18 groups on; with
PPVM_RUN_SCRATCH_MIN_GROUPS=1 every fused run with a group takes it.  The threshold is read
once per process, so the fused-run parity tests run again in a child process with it set:
the term lists must match the oracle's bit for bit, as in look-back mode."""

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
