"""GPU parity of the batched engine (PauliSumBatch -> ppvm_batch_* -> k_batch) against the oracle.

Every instance of a batch must equal the oracle's PauliSum run of the same list: the same
terms in the same order (IndexMap order), every coefficient bit for bit, and the same live
count entering every gate (term-gate updates).  overlap_with_zero is compared to 1e-10.
"""

import os
import sys

import numpy as np
import pytest

from ppvm_b200 import circuits as C
from ppvm_b200 import gates as G
from ppvm_b200.batch import Instance, PauliSumBatch
from tests.helpers import oracle_from
from tests.test_gpu_parity import _random_ops

pytestmark = pytest.mark.gpu


def oracle_of(inst: Instance, clifford_angles=False):
    o = oracle_from(inst.terms, inst.n_qubits, inst.min_abs_coeff, inst.max_pauli_weight, clifford_angles)
    cnt = o.run_ops(inst.ops, counts=True)
    return o, C.term_gate_updates(cnt, inst.ops)


def check_batch(b: PauliSumBatch, clifford_angles=False):
    owz = b.overlap_with_zero()
    per, total = b.term_gate_updates()
    want_total = 0
    for j, inst in enumerate(b.instances):
        o, tgu = oracle_of(inst, clifford_angles)
        gx, gz, gc = b.export(j)
        ox, oz, oc = o.export()
        assert gc.shape == oc.shape, (j, len(gc), len(oc))
        assert np.array_equal(gx, ox) and np.array_equal(gz, oz), j
        bad = np.nonzero(gc.view(np.uint64) != oc.view(np.uint64))[0]
        assert bad.size == 0, (j, bad[:5])
        assert abs(owz[j] - o.overlap_with_zero()) < 1e-10, j
        assert int(per[j]) == tgu, (j, int(per[j]), tgu)
        want_total += tgu
    assert total == want_total


def test_batched_tfim_matches_oracle_per_instance():
    wls = C.batched_tfim(count=24, seed=7)
    b = PauliSumBatch.from_workloads(wls)
    b.run()
    check_batch(b)
    b.run()  # a second run starts again from the initial terms
    check_batch(b)


def test_mixed_ops_widths_and_weight_caps():
    insts = []
    for n, seed in ((5, 1), (20, 2), (64, 3), (65, 4), (130, 5), (200, 6)):
        rng = np.random.default_rng(seed)
        hot = sorted(int(v) for v in rng.choice(n, min(n, 10), replace=False))
        terms = {}
        for _ in range(5):
            w = ["I"] * n
            for q in rng.choice(hot, 3, replace=False):
                w[int(q)] = "XYZ"[int(rng.integers(3))]
            terms["".join(w)] = float(rng.uniform(-1, 1))
        insts.append(Instance(n, list(terms.items()), _random_ops(rng, n, 120, hot), 1e-4, 8))
    b = PauliSumBatch(insts)
    b.run()
    check_batch(b)


def test_clifford_angles_and_growth_replay():
    # a kicked-Ising prefix (Clifford-angle RZZ layers) and an RX fan that outgrows its
    # initial 256-term region several times over
    k = C.kicked_ising_2d(L=4, layers=3, thr=1e-6, max_weight=None)
    fan = [G.r1(G.RX, q, 0.3) for q in range(11)] + [G.truncate(), G.truncate()]
    insts = [Instance(k.n_qubits, list(k.observable), list(k.ops), k.min_abs_coeff, None),
             Instance(11, [("Z" * 11, 1.0)], fan, 1e-9, None),
             Instance(3, [("ZII", 1.0)], [G.r1(G.RX, 0, 0.2), G.truncate()], 1e-9, None)]
    b = PauliSumBatch(insts, clifford_angles=True)
    b.run()
    assert b.len_of(1) == 2 ** 11
    check_batch(b, clifford_angles=True)


def test_configs_persistent_and_autotune_agree():
    wls = C.batched_tfim(count=12, seed=11)
    b = PauliSumBatch.from_workloads(wls)
    b.run()
    ref = [b.export(j) for j in range(len(b))]

    def same_as_ref():
        for j in range(len(b)):
            for u, v in zip(b.export(j), ref[j]):
                assert np.array_equal(np.asarray(u).view(np.uint64), np.asarray(v).view(np.uint64))

    for block, items, tf in ((128, 2, 2), (512, 4, 4), (256, 2, 4)):
        b.set_config(block, items, tf)
        b.run()
        same_as_ref()
    b.run_persistent()
    same_as_ref()
    cfg = b.autotune()
    assert cfg["block"] in (128, 256, 512) and cfg["best_ms"] > 0
    check_batch(b)


def test_rejects_bad_instances():
    with pytest.raises(ValueError):
        PauliSumBatch([Instance(4, [("ZIII", 1.0)], [G.g1(G.H, 4)])])
    with pytest.raises(ValueError):
        PauliSumBatch([Instance(4, [("ZIII", 1.0)], [G.g2(G.CNOT, 1, 1)])])


def test_noise_parameters_and_replaced_instances():
    # depolarising channels and repeated equal-valued ops (which share parameter entries),
    # then the same batch with one instance's list and terms replaced: its inputs are
    # uploaded again into the existing device block, and a later batch reuses the cached
    # buffers of this one
    rng = np.random.default_rng(21)
    n = 9
    hot = list(range(n))
    ops = []
    for i in range(60):
        q = int(rng.integers(n))
        k = i % 5
        if k == 0:
            ops.append(G.depolarize1(q, 0.01))
        elif k == 1:
            a, c = (int(v) for v in rng.choice(n, 2, replace=False))
            ops.append(G.depolarize2(a, c, 0.02))
        elif k == 2:
            ops.append(G.r1(G.RX, q, 0.4))
        elif k == 3:
            ops.append(G.pauli_error(q, (0.01, 0.02, 0.03)))
        else:
            ops.append(G.r2(G.RZZ, q, (q + 1) % n, -0.7))
        if i % 3 == 2:
            ops.append(G.truncate())
    insts = [Instance(n, [("Z" * n, 1.0), ("X" + "I" * (n - 1), 0.5)], ops, 1e-7, None),
             Instance(12, [("Z" + "I" * 11, 1.0)], _random_ops(rng, 12, 80, hot), 1e-6, 6)]
    b = PauliSumBatch(insts)
    b.run()
    check_batch(b)
    b.run()  # unchanged: replayed layer graphs
    check_batch(b)
    from ppvm_b200._lib import lib
    from ppvm_b200.paulisum import _p64, _pd, ops_array
    new_ops = _random_ops(rng, 12, 40, hot)
    gl = ops_array(new_ops)
    b._check(lib().ppvm_batch_set_ops(b._h, 1, gl.ptr, len(gl)))
    x, z = G.parse_word("IZ" + "I" * 10, 12)
    c = np.array([1.0])
    b._check(lib().ppvm_batch_add_terms(b._h, 1, _p64(x), _p64(z), _pd(c), 1))  # += into the terms
    b.instances[1] = Instance(12, [("Z" + "I" * 11, 1.0), ("IZ" + "I" * 10, 1.0)], new_ops, 1e-6, 6)
    b.run()
    check_batch(b)
    del b
    b2 = PauliSumBatch(insts)
    b2.run()
    check_batch(b2)


def test_bulk_setter_names_the_failing_instance():
    good = Instance(4, [("ZIII", 1.0)], [G.r1(G.RX, 0, 0.3), G.truncate()])
    bad = Instance(4, [("ZIII", 1.0)], [G.g1(G.H, 0), G.amplitude_damping(1, 0.1)])
    with pytest.raises(ValueError, match="instance 1"):
        PauliSumBatch([good, bad, good])
    b = PauliSumBatch([good, good])
    b.run()
    check_batch(b)


def test_batches_from_the_pool_match_the_oracle():
    # small instances run resident in shared memory by default; the same cases again with
    # PPVM_BATCH_RESIDENT=never (read once per process, so in a child process) run every
    # instance from the device pool
    import subprocess

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, PPVM_BATCH_RESIDENT="never")
    r = subprocess.run([sys.executable, "-m", "pytest", "tests/test_gpu_batch.py", "-m", "gpu", "-x", "-q",
                        "-k", "not from_the_pool"], cwd=root, env=env, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-2000:]
    assert " passed" in r.stdout
