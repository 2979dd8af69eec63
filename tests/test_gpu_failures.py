"""Failure handling on the GPU, made to happen without faulting anything.

Each case runs in a child process, because the settings it needs are read once per process:

- PPVM_SPIN_LIMIT: a look-back (the ordered compactions' wait for the tiles before it) gives
  up after that many polls.  At 1 poll, multi-tile compactions give up: the call returns
  PPVM_ETIMEOUT, the sum is marked unusable (later calls on it fail), and the CUDA context
  stays usable: a single-tile sum, whose look-backs never wait, still matches the oracle.
- PPVM_TEST_FAIL_ALLOC=growth: storage growth of a live sum fails as if the device had no
  memory left: the call returns PPVM_ECAPACITY, the sum is unusable, and a sum created with
  enough capacity runs the same circuit and matches the oracle.
- PPVM_TEST_FAIL_ALLOC=run-scratch with scratch mode forced: the fused runs cannot get their
  scratch planes and take look-back mode instead; the results still match the oracle.
- Scratch mode at its default threshold (2^18 groups) against look-back mode on a sum with
  millions of terms: bit-identical term lists and <O>.
"""

import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def child(script, env_extra, timeout=600):
    env = dict(os.environ, **env_extra)
    r = subprocess.run([sys.executable, "-c", script], cwd=ROOT, env=env, capture_output=True, text=True,
                       timeout=timeout)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


TIMEOUT_SCRIPT = r"""
import json
from ppvm_b200 import gates as G
from ppvm_b200._lib import PPVMError, ECUDA
from ppvm_b200.paulisum import PauliSum
from tests.helpers import oracle_from
from tests.test_gpu_parity import same
out = {"timeouts": 0, "poisoned_after_timeout": 0, "completed": 0, "completed_match": 0}
n = 22
ops = [G.r1(G.RX, q, 0.3) for q in range(n)] + [G.truncate()]
for attempt in range(4):
    s = PauliSum(["Z" * n], n, [1.0], min_abs_coeff=0.0, exact_order=True)
    try:
        s.run(ops)
    except PPVMError as e:
        if e.status == 4:  # PPVM_ETIMEOUT
            out["timeouts"] += 1
            try:
                s.overlap_with_zero()
            except PPVMError as e2:
                out["poisoned_after_timeout"] += e2.status == ECUDA
        continue
    out["completed"] += 1
    o = oracle_from([("Z" * n, 1.0)], n, thr=0.0)
    o.run_ops(ops)
    same(s, o)
    out["completed_match"] += 1
# one tile: no look-back ever waits
small = [G.r1(G.RX, q, 0.3) for q in range(8)] + [G.truncate()]
g = PauliSum(["Z" * 8], 8, [1.0], min_abs_coeff=0.0, exact_order=True)
g.run(small)
o = oracle_from([("Z" * 8, 1.0)], 8, thr=0.0)
o.run_ops(small)
same(g, o)
out["small_ok"] = abs(g.overlap_with_zero() - o.overlap_with_zero()) < 1e-12
print(json.dumps(out))
"""


def test_lookback_timeout_returns_status_and_poisons_only_that_sum():
    r = child(TIMEOUT_SCRIPT, {"PPVM_SPIN_LIMIT": "1"})
    assert r["timeouts"] >= 1, r
    assert r["poisoned_after_timeout"] == r["timeouts"], r
    assert r["completed_match"] == r["completed"], r
    assert r["small_ok"], r


GROWTH_SCRIPT = r"""
import json
from ppvm_b200 import gates as G
from ppvm_b200._lib import PPVMError
from ppvm_b200.paulisum import PauliSum
from tests.helpers import oracle_from
from tests.test_gpu_parity import same
n = 14
ops = [G.r1(G.RX, q, 0.3) for q in range(n)] + [G.truncate()]
out = {}
s = PauliSum(["Z" * n], n, [1.0], min_abs_coeff=1e-9, exact_order=True, capacity=1)
try:
    s.run(ops)
    out["first"] = 0
except PPVMError as e:
    out["first"] = e.status
try:
    s.overlap_with_zero()
    out["after"] = 0
except PPVMError as e:
    out["after"] = e.status
big = PauliSum(["Z" * n], n, [1.0], min_abs_coeff=1e-9, exact_order=True, capacity=1 << 15)
big.run(ops)
o = oracle_from([("Z" * n, 1.0)], n, thr=1e-9)
o.run_ops(ops)
same(big, o)
out["fresh_len"] = len(big)  # below 2^14: thr 1e-9 drops the smallest products
print(json.dumps(out))
"""


def test_failed_growth_returns_ecapacity():
    r = child(GROWTH_SCRIPT, {"PPVM_TEST_FAIL_ALLOC": "growth"})
    assert r["first"] == 2, r   # PPVM_ECAPACITY
    assert r["after"] == 3, r   # PPVM_ECUDA: the sum is in an error state
    assert r["fresh_len"] > 4096, r  # more than the first sum's capacity: it had to grow


def test_fused_runs_without_scratch_memory_fall_back_to_lookback_mode():
    env = dict(os.environ, PPVM_RUN_SCRATCH_MIN_GROUPS="1", PPVM_TEST_FAIL_ALLOC="run-scratch")
    r = subprocess.run([sys.executable, "-m", "pytest", "tests/test_gpu_parity.py", "-m", "gpu", "-x", "-q",
                        "-k", "fused or kicked or wide"],
                       cwd=ROOT, env=env, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-2000:]
    assert " passed" in r.stdout


MODES_SCRIPT = r"""
import hashlib, json
from ppvm_b200 import circuits as C
from ppvm_b200.paulisum import PauliSum
from tests.test_gpu_headline import layers_of
wl = C.kicked_ising_2d(L=12, layers=12, theta_h=0.6, thr=1e-7, max_weight=12)
s = PauliSum([wl.observable[0][0]], wl.n_qubits, [1.0], min_abs_coeff=wl.min_abs_coeff,
             max_pauli_weight=wl.max_weight, clifford_angles=True, capacity=1 << 22)
max_in, counts = 0, hashlib.sha256()
for layer in layers_of(wl.ops):
    entering = len(s)
    s.run(layer)
    counts.update(s.live_counts().tobytes())
    max_in = max(max_in, entering)
    if entering > 2_000_000:  # that layer's RX run had far more than 2^18 groups
        break
x, z, c = s.export()
terms = hashlib.sha256(x.tobytes() + z.tobytes() + c.tobytes()).hexdigest()
print(json.dumps({"len": len(s), "owz": s.overlap_with_zero().hex(), "max_in": max_in,
                  "terms": terms, "counts": counts.hexdigest()}))
"""


def test_scratch_mode_at_default_threshold_equals_lookback_mode():
    # scratch mode places the same terms at the same positions as look-back mode: the term
    # lists (in order), the live counts and <O> hash alike
    a = child(MODES_SCRIPT, {})
    b = child(MODES_SCRIPT, {"PPVM_RUN_SCRATCH_MIN_GROUPS": str(1 << 40)})
    assert a["max_in"] > 2_000_000, a
    assert a == b
