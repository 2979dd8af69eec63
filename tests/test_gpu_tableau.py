"""GPU parity of the composed Clifford pass (k_tableau) against the oracle, through the C ABI.

Runs of 8 or more Clifford gates take the tableau pass, with the TRUNCATE that follows them
fused in; noise channels split a run into tableau and per-op segments.  The term order is
kept, so exported term lists must equal the oracle's in order and bit for bit.
"""

import random

import numpy as np
import pytest

from ppvm_b200 import circuits as C
from ppvm_b200 import gates as G
from ppvm_b200.paulisum import PauliSum
from tests.helpers import oracle_from, planes
from tests.test_gpu_parity import gpu_from, run_both, same
from tests.test_tableau import random_clifford_ops

pytestmark = pytest.mark.gpu


def dense_terms(rng, n, k):
    terms = {}
    while len(terms) < k:
        terms["".join(rng.choice("IIXYZ") for _ in range(n))] = rng.uniform(-1, 1)
    return list(terms.items())


def mixed_ops(rng, n, blocks):
    ops = []
    for b in range(blocks):
        ops += random_clifford_ops(rng, n, rng.randrange(8, 90))
        if b % 3 == 1:
            ops.append(G.pauli_error(rng.randrange(n), (0.01, 0.02, 0.03)))
            ops += random_clifford_ops(rng, n, rng.randrange(1, 6))  # short: per-op pass
        ops.append(G.truncate())
    return ops


@pytest.mark.parametrize("n", [5, 64, 65, 130, 300, 512])
def test_tableau_runs_with_fused_truncation(n):
    rng = random.Random(n)
    terms = dense_terms(rng, n, 3000 if n > 5 else 200)
    maxw = max(2, (3 * n) // 5)
    run_both(terms, n, mixed_ops(rng, n, 6), thr=1e-3, maxw=maxw, clifford_angles=True, check_every=40)


def test_tableau_with_preserve_strings_keeps_the_strategy_separate():
    n = 10
    rng = random.Random(7)
    terms = dense_terms(rng, n, 400)
    keep = [w for w, _ in terms[:5]]
    g = PauliSum([w for w, _ in terms], n, [c for _, c in terms], min_abs_coeff=0.3, max_pauli_weight=4,
                 preserve_strings=keep, clifford_angles=True, exact_order=True)
    o = oracle_from(terms, n, thr=0.3, maxw=4, clifford_angles=True)
    o.set_preserve(*planes(keep, n))
    for _ in range(3):
        ops = random_clifford_ops(rng, n, 40) + [G.truncate()]
        g.run(ops)
        o.run_ops(ops)
        same(g, o)


def test_tableau_on_empty_and_tiny_sums():
    n = 9
    g = gpu_from([("XXXXXXXXX", 1e-6)], n, thr=1e-3)
    g.truncate()
    assert len(g) == 0
    g.run(random_clifford_ops(random.Random(1), n, 20) + [G.truncate()])
    assert len(g) == 0 and g.overlap_with_zero() == 0.0
    run_both([("ZIIIIIIIY", 0.5)], n, random_clifford_ops(random.Random(2), n, 30), thr=0.0,
             clifford_angles=True)


def test_tableau_live_counts_and_log():
    n = 40
    rng = random.Random(5)
    terms = dense_terms(rng, n, 500)
    ops = random_clifford_ops(rng, n, 50) + [G.truncate()] + random_clifford_ops(rng, n, 30)
    g = gpu_from(terms, n, thr=1e-2, maxw=12, clifford_angles=True)
    o = oracle_from(terms, n, thr=1e-2, maxw=12, clifford_angles=True)
    g.run(ops)
    want = o.run_ops(ops, counts=True)
    assert np.array_equal(g.live_counts(), want)
    same(g, o)


@pytest.mark.parametrize("trunc_between", [True, False])
def test_clifford_segment_folded_into_the_next_rx_run(trunc_between):
    # a Clifford segment (>= 8 ops) right before a fused RX run is applied inside the run's
    # passes; the replays after a group too large for the run (2^12 coordinates) and after a
    # capacity overflow must restart at the segment
    n = 12
    segment = [G.g1(G.H, q) for q in range(n)] + [G.g2(G.CNOT, q, q + 1) for q in range(n - 1)]
    rx = [G.r1(G.RX, q, 0.3 + 0.01 * q) for q in range(n)]
    ops = segment + ([G.truncate()] if trunc_between else []) + rx + [G.truncate()]
    for terms in ([("X" * n, 1.0)], [("XIXIXIXIXIXI", 0.5), ("ZZIIYYIIXXII", -0.25)]):
        for cap in (0, 1):
            g = gpu_from(terms, n, thr=1e-9, maxw=None, clifford_angles=True, capacity=cap, exact=False)
            o = oracle_from(terms, n, thr=1e-9, clifford_angles=True)
            g.run(ops)
            want = o.run_ops(ops, counts=True)
            from tests.test_gpu_parity import same_set
            same_set(g, o)
            assert np.array_equal(g.live_counts(), want)
            assert abs(g.overlap_with_zero() - o.overlap_with_zero()) < 1e-10


def test_folded_segment_with_weight_cap_keeps_counts():
    wl = C.kicked_ising_2d(L=6, layers=5, thr=1e-5, max_weight=6)
    g = gpu_from(wl.observable, wl.n_qubits, wl.min_abs_coeff, wl.max_weight, True, exact=False)
    o = oracle_from(wl.observable, wl.n_qubits, wl.min_abs_coeff, wl.max_weight, True)
    g.run(wl.ops)
    want = o.run_ops(wl.ops, counts=True)
    from tests.test_gpu_parity import same_set
    same_set(g, o)
    assert np.array_equal(g.live_counts(), want)


def heavy_and_light_terms(rng, n, k):
    # light terms first (at most 3 non-identity qubits), heavy ones after: warps of light
    # terms keep the per-generator product, warps of heavy ones take the chunk tables
    terms = {}
    while len(terms) < k // 2:
        w = ["I"] * n
        for q in rng.sample(range(n), rng.randrange(1, 4)):
            w[q] = rng.choice("XYZ")
        terms["".join(w)] = rng.uniform(-1, 1)
    while len(terms) < k:
        terms["".join(rng.choice("IXYZ") for _ in range(n))] = rng.uniform(-1, 1)
    return list(terms.items())


@pytest.mark.parametrize("n", [40, 64])
def test_tableau_chunk_tables_on_large_one_word_sums(n):
    # 40,000 terms of one word through runs that move most generators: the pass builds the
    # chunk tables (from 2^15 terms on), and mixed warps choose per warp
    rng = random.Random(100 + n)
    terms = heavy_and_light_terms(rng, n, 40000)
    ops = []
    for _ in range(3):
        ops += random_clifford_ops(rng, n, 120) + [G.truncate()]
    run_both(terms, n, ops, thr=1e-4, maxw=None, clifford_angles=True, check_every=121)

