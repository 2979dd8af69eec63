"""The composed Clifford pass with its chunk tables forced on and off, against the oracle.

One-word sums (n <= 64) of 2^15 terms or more, through a run that moves 32 generators or
more, map through per-chunk image tables; PPVM_TABLEAU_CHUNKS=always|never forces the choice
(read once per process), so the tableau parity cases run again in a child process with each
set.  The child selects tests of the two parity files only, never of this file."""

import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def rerun(mode, select):
    env = dict(os.environ, PPVM_TABLEAU_CHUNKS=mode)
    r = subprocess.run([sys.executable, "-m", "pytest", "tests/test_gpu_tableau.py", "tests/test_gpu_parity.py",
                        "-m", "gpu", "-x", "-q", "-k", select],
                       cwd=ROOT, env=env, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-2000:]
    assert " passed" in r.stdout


def test_tableau_cases_with_chunk_tables_forced():
    # every one-word tableau pass with a moved generator takes the tables, light terms too
    rerun("always", "tableau or clifford_t or kicked or folded or segment")


def test_large_one_word_sums_without_chunk_tables():
    rerun("never", "chunk_tables_on_large or clifford_t")
