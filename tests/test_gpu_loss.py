"""Lossy sums (LossyPauliWord) on the GPU against the oracle, through the C ABI.

The oracle restates the reference's loss semantics literally (its own loss plane and the
reference's per-gate loss checks, pinned by tests/test_oracle_loss.py); the engine keeps the
loss bits in the X plane's upper words and masks generators and two-qubit gates per term.
Term lists must match bit for bit: in order with ``exact_order``, as sets otherwise.
"""

import json
import os

import numpy as np
import pytest

from ppvm_b200 import gates as G
from ppvm_b200.paulisum import LossyPauliSum
from tests.helpers import lossy_list, lossy_oracle_from

pytestmark = pytest.mark.gpu
GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_tables.json")))
OPS = {"x": G.X, "y": G.Y, "z": G.Z, "h": G.H, "s": G.S, "s_dag": G.S_DAG, "sqrt_x": G.SQRT_X,
       "sqrt_x_dag": G.SQRT_X_DAG, "sqrt_y": G.SQRT_Y, "sqrt_y_dag": G.SQRT_Y_DAG, "cnot": G.CNOT,
       "cz": G.CZ, "cy": G.CY}


def gpu(terms, n, thr=0.0, maxw=None, max_loss_weight=None, exact=True, clifford_angles=False, capacity=0):
    return LossyPauliSum([w for w, _ in terms], n, [c for _, c in terms], min_abs_coeff=thr, max_pauli_weight=maxw,
                         max_loss_weight=max_loss_weight, exact_order=exact, clifford_angles=clifford_angles,
                         capacity=capacity)


def same(g, o, exact=True):
    gx, gz, gc = g.export()
    ox, oz, oc = o.export()
    assert len(gc) == len(oc), (len(gc), len(oc))
    gk = np.concatenate([gx, gz, gc.view(np.uint64)[:, None]], axis=1)
    ok = np.concatenate([ox, oz, oc.view(np.uint64)[:, None]], axis=1)
    if not exact:
        gk = gk[np.lexsort(gk.T[::-1])] if len(gc) else gk
        ok = ok[np.lexsort(ok.T[::-1])] if len(oc) else ok
    bad = np.nonzero((gk != ok).any(axis=1))[0]
    assert bad.size == 0, (bad[:5], [lossy_list(o)[i] for i in bad[:3]], [g.terms[i] for i in bad[:3]])


@pytest.mark.parametrize("name", sorted(GOLD["loss_word_tables"]))
def test_lossy_clifford_tables(name):
    # crates/ppvm-pauli-word/src/loss/clifford.rs:13-207
    for inp, out in GOLD["loss_word_tables"][name]:
        n = len(inp)
        s = gpu([(inp, 1.0)], n)
        s.run([G.g1(OPS[name], 0)] if n == 1 else [G.g2(OPS[name], 0, 1)])
        assert [w for w, _ in s.terms] == [out], (name, inp)


def test_reference_loss_cases():
    # crates/ppvm-pauli-sum/tests/loss.rs through the Python-style API
    s = gpu([("I", 2.0), ("Z", 3.0)], 1)
    s.reset_loss_channel(0)
    assert s.terms == [("I", 2.0), ("Z", 3.0), ("L", 5.0)]
    s = gpu([("L", 1.0)], 1)
    s.loss_channel(0, 0.2)
    assert dict(s.terms) == {"L": 1.0, "I": 0.2}
    for w in "XYIZ":
        s = gpu([(w, 1.0)], 1)
        s.loss_channel(0, 0.2)
        assert s.terms == [(w, 0.8)]
    p = [0.1, 0.05, 0.2]
    s = gpu([("LL", 1.0)], 2)
    s.correlated_loss_channel(0, 1, p)
    assert s.terms == [("IL", p[2]), ("LI", p[2]), ("II", p[0]), ("LL", 1.0)]  # children order first
    s = gpu([("ZZ", 1.0)], 2)
    for q in (0, 1):
        s.reset_loss_channel(q)
    for q in (0, 1):
        s.loss_channel(q, 0.1)
    s.cnot(0, 1)
    s.h(0)
    prob = 0.5 + 0.5 * ((1.0 - 0.1) * (1.0 - 0.1) - 2.0 * 0.1 * (1.0 - 0.1) + 0.1 * 0.1)
    assert abs(s.overlap_with_zero() - prob) < 1e-10 and abs(s.trace("Z?*") - prob) < 1e-10
    s = gpu([("ZZZ", 1.0)], 3, max_loss_weight=2)
    for q in range(3):
        s.reset_loss_channel(q, truncate=False)
    for q in range(3):
        s.loss_channel(q, 0.1, truncate=False)
    before = len(s)
    s.truncate()
    assert len(s) == before - 1 and "LLL" not in dict(s.terms)


def random_lossy_terms(rng, n, m, max_w=5):
    terms = {}
    while len(terms) < m:
        w = ["I"] * n
        for q in rng.choice(n, int(rng.integers(1, min(max_w, n) + 1)), replace=False):
            w[int(q)] = "XYZLL"[int(rng.integers(5))]
        terms["".join(w)] = float(rng.uniform(-1, 1))
    return list(terms.items())


def random_lossy_ops(rng, n, count, hot):
    one = [G.X, G.Y, G.Z, G.H, G.S, G.S_DAG, G.SQRT_X, G.SQRT_X_DAG, G.SQRT_Y, G.SQRT_Y_DAG]
    pick = lambda: int(rng.choice(hot))  # noqa: E731

    def pair():
        a, b = (int(v) for v in rng.choice(hot, 2, replace=False))
        return a, b

    ops = []
    for i in range(count):
        k = int(rng.integers(0, 14))
        if k < 2:
            ops.append(G.g1(int(rng.choice(one)), pick()))
        elif k < 4:
            ops.append(G.g2(int(rng.choice([G.CNOT, G.CZ, G.CY])), *pair()))
        elif k < 6:
            ops.append(G.r1(int(rng.choice([G.RX, G.RY, G.RZ])), pick(), float(rng.uniform(-3, 3))))
        elif k < 8:
            ops.append(G.r2(int(rng.choice([G.RXX, G.RYY, G.RZZ])), *pair(), float(rng.uniform(-3, 3))))
        elif k == 8:
            ops.append(G.loss_channel(pick(), float(rng.uniform(0, 0.3))))
        elif k == 9:
            ops.append(G.reset_loss_channel(pick()))
        elif k == 10:
            ops.append(G.correlated_loss_channel(*pair(), rng.uniform(0, 0.2, 3)))
        elif k == 11:
            ops.append(G.depolarize2(*pair(), float(rng.uniform(0, 0.1))))
        elif k == 12:
            ops.append(G.amplitude_damping(pick(), float(rng.uniform(0, 0.3))))
        else:
            ops.append(G.pauli_error(pick(), rng.uniform(0, 0.05, 3)))
        if i % 4 == 3:
            ops.append(G.truncate())
    return ops


@pytest.mark.parametrize("exact", [True, False])
@pytest.mark.parametrize("n", [3, 20, 64, 65, 130, 256])
def test_random_lossy_circuits(n, exact):
    rng = np.random.default_rng(700 + n)
    hot = sorted(int(v) for v in rng.choice(n, min(n, 10), replace=False))
    terms = random_lossy_terms(rng, n, min(200, 3 ** n // 2))
    ops = random_lossy_ops(rng, n, 200, hot)
    g = gpu(terms, n, thr=1e-4, maxw=9, max_loss_weight=3, exact=exact, capacity=1)
    o = lossy_oracle_from(terms, n, thr=1e-4, maxw=9, max_loss_weight=3)
    for i in range(0, len(ops), 10):
        g.run(ops[i:i + 10])
        want = o.run_ops(ops[i:i + 10], counts=True)
        assert np.array_equal(g.live_counts(), want)
        same(g, o, exact)
    assert abs(g.overlap_with_zero() - o.overlap_with_zero()) < 1e-10
    for pat in ("Z?*", "[XY]*", f"Z{hot[0]}"):
        assert abs(g.trace(pat) - o.trace(pat)) < 1e-10


@pytest.mark.parametrize("exact", [True, False])
def test_lossy_runs_tableau_and_clifford_angles(exact):
    # long Clifford stretches (the composed pass takes the one-qubit gates, the per-op pass the
    # two-qubit ones), fused RX runs and Clifford-angle RZZ on a lossy sum
    n = 40
    rng = np.random.default_rng(11)
    terms = random_lossy_terms(rng, n, 300, max_w=4)
    ops = []
    for layer in range(3):
        ops += [G.g1(int(rng.choice([G.H, G.S, G.S_DAG, G.SQRT_X])), q) for q in range(n)]
        ops += [G.g2(G.CNOT, q, q + 1) for q in range(0, n - 1, 2)]
        ops += [G.r2(G.RZZ, q, q + 1, -np.pi / 2) for q in range(1, n - 1, 2)] + [G.truncate()]
        ops += [G.r1(G.RX, q, 0.3) for q in range(n)] + [G.truncate()]
        ops += [G.reset_loss_channel(int(q)) for q in rng.choice(n, 3, replace=False)]
        ops += [G.correlated_loss_channel(2 * layer, 2 * layer + 1, [0.05, 0.02, 0.1])] + [G.truncate()]
    g = gpu(terms, n, thr=1e-3, maxw=8, exact=exact, clifford_angles=True)
    o = lossy_oracle_from(terms, n, thr=1e-3, maxw=8, clifford_angles=True)
    for i in range(0, len(ops), 40):
        g.run(ops[i:i + 40])
        o.run_ops(ops[i:i + 40])
        same(g, o, exact)


def test_correlated_channel_keeps_the_larger_maps_order():
    # many (L,L) terms: more distinct children than terms, so the children's order leads
    n = 6
    terms = [(w, 0.5 + 0.1 * i) for i, w in enumerate(["LLXIII", "LLIZII", "LLIIYI", "IILLII", "LXIIII"])]
    for pair in ((0, 1), (2, 3), (1, 2)):
        g = gpu(terms, n)
        o = lossy_oracle_from(terms, n)
        g.correlated_loss_channel(*pair, [0.1, 0.05, 0.2], truncate=False)
        o.run_ops([G.correlated_loss_channel(*pair, [0.1, 0.05, 0.2])])
        same(g, o)


def test_lossy_capacity_growth_and_words():
    # reset on every qubit doubles the sum per qubit: growth and replay inside loss ops
    n = 14
    g = gpu([("Z" * n, 1.0)], n, capacity=1)
    o = lossy_oracle_from([("Z" * n, 1.0)], n)
    ops = [G.reset_loss_channel(q) for q in range(n)] + [G.loss_channel(q, 0.1) for q in range(n)]
    g.run(ops)
    o.run_ops(ops)
    same(g, o)
    assert len(g) > 4096
    with pytest.raises(ValueError):
        LossyPauliSum(["Q"], 1)
    with pytest.raises(ValueError):
        LossyPauliSum(["Z" * 300], 300)
