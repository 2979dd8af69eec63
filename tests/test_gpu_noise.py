"""GPU parity of the two-qubit Pauli error and amplitude damping against the oracle.

Coefficients must match bit for bit.  With ``exact_order`` the term order must match too;
the reference's map_insert appends new children after all terms, in parent order.
"""

import ctypes
import math

import numpy as np
import pytest

from ppvm_b200 import gates as G
from ppvm_b200._lib import OK, lib
from ppvm_b200.paulisum import PauliSum
from tests.helpers import oracle_dict, oracle_from
from tests.test_gpu_parity import gpu_from, same, same_set

pytestmark = pytest.mark.gpu


def random_terms(rng, n, m, max_w=5):
    max_w = min(max_w, n)
    m = min(m, (4 ** n - 1) // 2)  # leave room: small n has few words
    terms = {}
    while len(terms) < m:
        w = ["I"] * n
        for q in rng.choice(n, int(rng.integers(1, max_w + 1)), replace=False):
            w[int(q)] = "XYZ"[int(rng.integers(3))]
        terms["".join(w)] = float(rng.uniform(-1, 1))
    return list(terms.items())


def test_two_qubit_pauli_error_known_answers():
    # crates/ppvm-pauli-sum/tests/noise.rs:8-95
    p = [0.0] * 15
    p[0] = 1.0
    s = gpu_from([("IZ", 1.0)], 2)
    s.two_qubit_pauli_error([0, 1], p, truncate=False)
    assert s.terms == [("IZ", -1.0)]
    p = [0.0] * 15
    p[4], p[14] = 1.0, 1.0
    s = gpu_from([("XI", 1.0)], 2)
    s.two_qubit_pauli_error(0, 1, p)
    assert s.terms == [("XI", -1.0)]


@pytest.mark.parametrize("n", [3, 64, 65, 130])
def test_two_qubit_pauli_error_parity(n):
    rng = np.random.default_rng(n)
    terms = random_terms(rng, n, 400)
    pairs = []
    for _ in range(6):
        a, b = (int(v) for v in rng.choice(n, 2, replace=False))
        pairs += [a, b]
    p = rng.uniform(0, 1 / 15, 15)
    for truncate in (False, True):
        g = gpu_from(terms, n, thr=0.05)
        o = oracle_from(terms, n, thr=0.05)
        g.two_qubit_pauli_error(pairs, p, truncate=truncate)
        o.two_qubit_pauli_error(pairs, p, truncate=truncate)
        same(g, o)
    with pytest.raises(ValueError):
        gpu_from(terms, n).two_qubit_pauli_error(pairs[:-1], p)
    with pytest.raises(ValueError):
        gpu_from(terms, n).two_qubit_pauli_error([1, 1], p)


def test_amplitude_damping_known_answers():
    # crates/ppvm-pauli-sum/tests/noise.rs:223-265
    g = 0.3
    s = gpu_from([("ZI", 1.0)], 2)
    s.amplitude_damping(0, g)
    assert s.terms == [("ZI", 1.0 - g), ("II", 1.0 * g)]
    s = gpu_from([("XI", 1.0)], 2)
    s.amplitude_damping(0, g)
    assert s.terms == [("XI", math.sqrt(1.0 - g))]
    s = gpu_from([("II", 1.0)], 2)
    s.amplitude_damping(0, g)
    assert s.terms == [("II", 1.0)]


@pytest.mark.parametrize("n", [4, 64, 100, 200])
def test_amplitude_damping_parity(n):
    rng = np.random.default_rng(10 + n)
    terms = random_terms(rng, n, 600, max_w=4)
    # partners: for some Z-on-q terms add the same word with I on q
    q = int(rng.integers(n))
    extra = {}
    for w, c in terms[:200]:
        lst = list(w)
        lst[q] = "Z"
        extra["".join(lst)] = c
        lst[q] = "I"
        extra["".join(lst)] = -0.5 * c
    terms = list(dict(terms + list(extra.items())).items())
    for exact in (True, False):
        gs = gpu_from(terms, n, thr=1e-3, exact=exact)
        o = oracle_from(terms, n, thr=1e-3)
        ops = [G.amplitude_damping(q, 0.2), G.r1(G.RX, q, 0.3), G.amplitude_damping(q, 0.7), G.truncate()]
        ops += [G.amplitude_damping(int(rng.integers(n)), float(rng.uniform())) for _ in range(5)]
        ops += [G.truncate()]
        gs.run(ops)
        o.run_ops(ops)
        (same if exact else same_set)(gs, o)
        assert abs(gs.overlap_with_zero() - o.overlap_with_zero()) < 1e-10


def test_amplitude_damping_grows_and_replays_without_rescaling():
    # 5000 Z-on-0 parents with no partners double the sum past its capacity: the op stops
    # before touching any coefficient, grows, and replays; X/Y terms are scaled once
    n = 40
    rng = np.random.default_rng(3)
    terms = {}
    while len(terms) < 6000:
        w = ["I"] * n
        w[0] = "Z" if len(terms) < 5000 else "XY"[len(terms) % 2]
        for q in rng.choice(np.arange(1, n), 3, replace=False):
            w[int(q)] = "XYZ"[int(rng.integers(3))]
        terms["".join(w)] = float(rng.uniform(-1, 1))
    terms = list(terms.items())
    assert lib().ppvm_release_cached_memory() == OK  # a fresh handle: 8192 terms after the load
    g = gpu_from(terms, n, thr=1e-12, exact=True)
    o = oracle_from(terms, n, thr=1e-12)
    g.amplitude_damping(0, 0.35)
    o.run_ops([G.amplitude_damping(0, 0.35), G.truncate()])
    same(g, o)
    assert len(g) == 11000


def test_amplitude_damping_in_fused_lists():
    # damping between fused RX runs and Clifford stretches of a gate list
    n = 36
    rng = np.random.default_rng(5)
    terms = random_terms(rng, n, 50, max_w=3)
    ops = []
    for layer in range(3):
        ops += [G.r1(G.RX, q, 0.4) for q in range(n)] + [G.truncate()]
        ops += [G.amplitude_damping(q, 0.1 + 0.05 * layer) for q in range(0, n, 5)]
        ops += [G.g2(G.CNOT, q, q + 1) for q in range(0, n - 1, 2)] + [G.truncate()]
    g = gpu_from(terms, n, thr=1e-4, maxw=6, exact=False)
    o = oracle_from(terms, n, thr=1e-4, maxw=6)
    g.run(ops)
    o.run_ops(ops)
    same_set(g, o)


def test_batch_rejects_amplitude_damping():
    from ppvm_b200.batch import Instance, PauliSumBatch

    inst = Instance(n_qubits=4, terms=[("ZIII", 1.0)], ops=[G.amplitude_damping(0, 0.1)])
    with pytest.raises(ValueError):
        PauliSumBatch([inst])


@pytest.mark.parametrize("exact", [True, False])
@pytest.mark.parametrize("n", [3, 64, 65, 200])
def test_depolarize_parity(n, exact):
    # Depolarizing::depolarize1 / depolarize2 (crates/ppvm-pauli-sum/src/sum/noise.rs:107-129):
    # every term with a non-identity Pauli on the target(s) is scaled, between rotations that
    # keep the sum changing, with truncations that drop scaled terms
    rng = np.random.default_rng(300 + n)
    terms = random_terms(rng, n, 300)
    hot = [int(v) for v in rng.choice(n, min(n, 8), replace=False)]
    ops = []
    for k in range(6):
        a, b = hot[k % len(hot)], hot[(k + 1) % len(hot)]
        ops += [G.r1(G.RX, a, 0.3 + 0.1 * k), G.depolarize1(a, 0.01 * (k + 1)), G.depolarize1(b, 0.2),
                G.r2(G.RZZ, a, b, -0.4), G.depolarize2(a, b, 0.03 * (k + 1)), G.truncate()]
    g = gpu_from(terms, n, thr=2e-3, exact=exact)
    o = oracle_from(terms, n, thr=2e-3)
    for i in range(0, len(ops), 6):
        g.run(ops[i:i + 6])
        o.run_ops(ops[i:i + 6])
        (same if exact else same_set)(g, o)
    # the per-gate entry points with their own truncate flag
    g2 = gpu_from(terms, n, thr=0.05, exact=True)
    o2 = oracle_from(terms, n, thr=0.05)
    pairs = hot[:4] if len(hot) >= 4 else hot[:2]
    g2.depolarize1(hot[:3], p=0.3)
    g2.depolarize2(pairs, p=0.4, truncate=False)
    o2.run_ops([G.depolarize1(q, 0.3) for q in hot[:3]] + [G.truncate()])
    o2.run_ops([G.depolarize2(pairs[i], pairs[i + 1], 0.4) for i in range(0, len(pairs), 2)])
    same(g2, o2)
