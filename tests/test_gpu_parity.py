"""GPU engine vs the CPU oracle, through the C ABI (ppvm_b200.PauliSum -> libppvm_cuda.so).

Two modes are checked.  With ``exact_order`` the engine keeps the reference's term order
(IndexMap order) and the exported term lists must be identical, word for word and
coefficient bit for bit.  In the default mode fused rotation runs reorder terms, so the
sorted term lists must be identical, again with every coefficient equal bit for bit.
overlap_with_zero sums in a different order than the reference's sequential fold, so it is
compared to 1e-10 absolute.
"""

import json
import math
import os

import numpy as np
import pytest

from ppvm_b200 import circuits as C
from ppvm_b200 import gates as G
from ppvm_b200.paulisum import PauliSum
from tests.helpers import oracle_from, oracle_list, planes

pytestmark = pytest.mark.gpu
GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_tables.json")))


def gpu_from(terms, n, thr=1e-10, maxw=None, clifford_angles=False, capacity=0, preserve=None,
             exact=True):
    return PauliSum([t for t, _ in terms], n, [c for _, c in terms], min_abs_coeff=thr,
                    max_pauli_weight=maxw, preserve_strings=preserve, clifford_angles=clifford_angles,
                    capacity=capacity, exact_order=exact)


def same(gpu, orc):
    """Identical term lists: same words in the same order, coefficients equal bit for bit."""
    gx, gz, gc = gpu.export()
    ox, oz, oc = orc.export()
    assert gc.shape == oc.shape, (len(gc), len(oc))
    assert np.array_equal(gx, ox) and np.array_equal(gz, oz)
    bad = np.nonzero(gc.view(np.uint64) != oc.view(np.uint64))[0]
    assert bad.size == 0, (bad[:5], gc[bad[:5]], oc[bad[:5]])


def _sorted(x, z, c):
    keys = np.concatenate([x, z], axis=1)
    order = np.lexsort(keys.T[::-1]) if len(c) else np.zeros(0, dtype=np.int64)
    return keys[order], c[order]


def same_set(gpu, orc):
    """Identical term sets, every coefficient equal bit for bit (order free)."""
    gk, gc = _sorted(*gpu.export())
    ok, oc = _sorted(*orc.export())
    assert gc.shape == oc.shape, (len(gc), len(oc))
    assert np.array_equal(gk, ok)
    bad = np.nonzero(gc.view(np.uint64) != oc.view(np.uint64))[0]
    assert bad.size == 0, (bad[:5], gc[bad[:5]], oc[bad[:5]])


def run_both(terms, n, ops, thr=1e-10, maxw=None, clifford_angles=False, capacity=0, check_every=None,
             exact=True):
    g = gpu_from(terms, n, thr, maxw, clifford_angles, capacity, exact=exact)
    o = oracle_from(terms, n, thr, maxw, clifford_angles)
    step = check_every or max(1, len(ops))
    for i in range(0, len(ops), step):
        chunk = ops[i:i + step]
        g.run(chunk)
        o.run_ops(chunk)
        (same if exact else same_set)(g, o)
    assert abs(g.overlap_with_zero() - o.overlap_with_zero()) < 1e-10
    return g, o


def test_cnot_golden():
    ops = [G.r1(G.RZ, 0, 1.1), G.r1(G.RY, 0, 2.1), G.r1(G.RZ, 0, 1.1), G.r1(G.RZ, 1, 1.1),
           G.r1(G.RY, 1, 2.1), G.r1(G.RZ, 1, 1.1), G.g2(G.CNOT, 0, 1), G.r1(G.RX, 0, 2.1),
           G.r1(G.RX, 1, 2.1)]
    g, _ = run_both([("ZZ", 1.0)], 2, ops, thr=0.0, check_every=1)
    assert math.isclose(g.trace("Z?*"), GOLD["golden_cnot"], rel_tol=1e-12)


def test_trotter_golden():
    n = 4
    seed = [(C._z_word(n, j), 1.0) for j in range(n)]
    ops = []
    for _ in range(10):
        for i in range(n):
            ops += [G.pauli_error(i, (2.5e-5,) * 3), G.truncate(), G.r1(G.RX, i, 0.1), G.truncate()]
        for i in range(n - 1):
            ops += [G.pauli_error(i + 1, (2.5e-5,) * 3), G.truncate(), G.pauli_error(i, (2.5e-5,) * 3),
                    G.truncate(), G.r2(G.RZZ, i, i + 1, 0.0125), G.truncate()]
    g, _ = run_both(seed, n, ops, thr=0.0, check_every=7)
    ev = sum(c for w, c in g.terms if set(w) <= {"I", "Z"})
    assert abs(ev - GOLD["golden_trotter_n4"]) < 1e-9


@pytest.mark.parametrize("name", sorted(GOLD["phase_tables"]))
def test_clifford_sign_tables(name):
    code = {"x": G.X, "y": G.Y, "z": G.Z, "h": G.H, "s": G.S, "s_dag": G.S_DAG, "sqrt_x": G.SQRT_X,
            "sqrt_x_dag": G.SQRT_X_DAG, "sqrt_y": G.SQRT_Y, "sqrt_y_dag": G.SQRT_Y_DAG,
            "cnot": G.CNOT, "cz": G.CZ, "cy": G.CY}[name]
    for inp, out in GOLD["phase_tables"][name]:
        si = -1.0 if inp[0] == "-" else 1.0
        wi = inp.lstrip("+-")
        so = -1.0 if out[0] == "-" else 1.0
        n = len(wi)
        g = gpu_from([(wi, si)], n, thr=0.0)
        g.run([G.g1(code, 0)] if n == 1 else [G.g2(code, 0, 1)])
        assert g.terms == [(out.lstrip("+-"), so * si)]


def test_rot_children_exact():
    t = 2.1
    for code in (G.RX, G.RY, G.RZ):
        for w in "IXYZ":
            run_both([(w, 1.0)], 1, [G.r1(code, 0, t)], thr=0.0)
    for code in (G.RXX, G.RYY, G.RZZ):
        for p in "IXYZ":
            for q in "IXYZ":
                run_both([(p + "I" + q, 1.0)], 3, [G.r2(code, 0, 2, 0.7)], thr=0.0)


def _random_ops(rng, n, count, hot):
    """Random gates on a small hot qubit set spread over the words, TRUNCATE every 4 ops, so
    the term count stays bounded (at most 2^4 growth between truncations)."""
    ops = []
    one = [G.X, G.Y, G.Z, G.H, G.S, G.S_DAG, G.SQRT_X, G.SQRT_X_DAG, G.SQRT_Y, G.SQRT_Y_DAG]
    pick = lambda: int(rng.choice(hot))  # noqa: E731

    def pair():
        a, b = (int(v) for v in rng.choice(hot, 2, replace=False))
        return a, b

    for i in range(count):
        k = rng.integers(0, 9)
        if k < 2:
            ops.append(G.g1(int(rng.choice(one)), pick()))
        elif k < 3:
            ops.append(G.g2(int(rng.choice([G.CNOT, G.CZ, G.CY])), *pair()))
        elif k < 6:
            ops.append(G.r1(int(rng.choice([G.RX, G.RY, G.RZ])), pick(), float(rng.uniform(-3, 3))))
        elif k < 8:
            ops.append(G.r2(int(rng.choice([G.RXX, G.RYY, G.RZZ])), *pair(), float(rng.uniform(-3, 3))))
        else:
            ops.append(G.pauli_error(pick(), rng.uniform(0, 0.05, 3)))
        if i % 4 == 3:
            ops.append(G.truncate())
    return ops


def random_case(n, seed):
    rng = np.random.default_rng(seed)
    hot = sorted(int(v) for v in rng.choice(n, min(n, 12), replace=False))
    terms = {}
    for _ in range(6):
        w = ["I"] * n
        for q in rng.choice(hot, 3, replace=False):
            w[int(q)] = "XYZ"[int(rng.integers(3))]
        terms["".join(w)] = float(rng.uniform(-1, 1))
    return list(terms.items()), _random_ops(rng, n, 160, hot)


@pytest.mark.parametrize("exact", [True, False])
@pytest.mark.parametrize("n", [5, 20, 64, 65, 100, 144, 200])
def test_random_circuits(n, exact):
    terms, ops = random_case(n, n)
    g, _ = run_both(terms, n, ops, thr=1e-4, maxw=8, check_every=10, exact=exact)


@pytest.mark.parametrize("n", [12, 70, 144, 200])
def test_fused_rotation_runs(n):
    # layers of RX on every qubit then RZ on every qubit (each a fused run ending in TRUNCATE),
    # with Clifford layers in between; sparse random start terms
    rng = np.random.default_rng(100 + n)
    terms = {}
    for _ in range(20):
        w = ["I"] * n
        for q in rng.choice(n, 3, replace=False):
            w[int(q)] = "XYZ"[int(rng.integers(3))]
        terms["".join(w)] = float(rng.uniform(-1, 1))
    ops = []
    for layer in range(3):
        ops += [G.r1(G.RX, q, 0.3 + 0.01 * layer) for q in rng.permutation(n)] + [G.truncate()]
        ops += [G.g2(G.CNOT, q, q + 1) for q in range(0, n - 1, 2)]
        ops += [G.r1(G.RZ, q, -0.7) for q in range(n)]  # no TRUNCATE: run without a cut
        ops += [G.g1(G.H, q) for q in range(0, n, 3)] + [G.truncate()]
    run_both(list(terms.items()), n, ops, thr=1e-3, maxw=6, check_every=len(ops) // 3, exact=False)


def test_capacity_growth_replay():
    # Z^14 through RX on every qubit without truncation branches to exactly 2^14 terms,
    # beyond the initial 4096-term capacity: rotations overflow, grow and replay.
    n = 14
    ops = [G.r1(G.RX, q, 0.3) for q in range(n)] + [G.r1(G.RZ, q, 0.4) for q in range(3)] + [G.truncate()]
    for exact in (True, False):  # fused: |M| = 14 > 10 falls back to the per-gate path
        g = gpu_from([("Z" * n, 1.0)], n, thr=1e-9, capacity=1, exact=exact)
        o = oracle_from([("Z" * n, 1.0)], n, thr=1e-9)
        g.run(ops)
        o.run_ops(ops)
        (same if exact else same_set)(g, o)
        assert len(g) > 4096


def test_wide_run_splits_until_it_fits():
    # Z on qubits 0..11 meets a 40-gate RX run in qubit order: 12 > 10 coordinates.  The
    # group keeps them through the whole run, so after its 2nd coordinate (gate 1) at most 10
    # remain: gates 0 and 1 replay one at a time and gates 2..39 fuse.  The RZ and RX layers
    # after it meet wide groups again on a larger sum
    n = 40
    rng = np.random.default_rng(7)
    terms = {"Z" * 12 + "I" * (n - 12): 1.0}
    for _ in range(30):
        w = ["I"] * n
        for q in rng.choice(n, 4, replace=False):
            w[int(q)] = "XYZ"[int(rng.integers(3))]
        terms["".join(w)] = float(rng.uniform(-1, 1))
    ops = [G.r1(G.RX, q, 0.4) for q in range(n)] + [G.truncate()]
    ops += [G.r1(G.RZ, q, 0.3) for q in range(n)] + [G.truncate()]
    ops += [G.r1(G.RX, q, -0.2) for q in range(n)] + [G.truncate()]
    run_both(list(terms.items()), n, ops, thr=1e-6, check_every=n + 1, exact=False)


def test_wide_run_fuses_its_tail():
    # Z on qubits 20..31 meets a 32-gate RX run in qubit order: the first 22 gates (up to its
    # 2nd coordinate) go one at a time and the last 10 fuse
    n = 32
    terms = [("I" * 20 + "Z" * 12, 1.0), ("X" + "I" * 30 + "Y", -0.5), ("IZ" + "I" * 30, 0.25)]
    ops = [G.r1(G.RX, q, 0.35) for q in range(n)] + [G.truncate()]
    run_both(terms, n, ops, thr=1e-7, exact=False)


@pytest.mark.parametrize("exact", [True, False])
def test_tfim_config1_every_half(exact):
    wl = C.tfim_1d()
    run_both(wl.observable, wl.n_qubits, wl.ops, thr=wl.min_abs_coeff, check_every=20, exact=exact)


@pytest.mark.parametrize("exact", [True, False])
def test_kicked_ising_prefix(exact):
    wl = C.kicked_ising_2d(layers=4)
    g, o = run_both(wl.observable, wl.n_qubits, wl.ops, thr=wl.min_abs_coeff, maxw=wl.max_weight,
                    clifford_angles=True, check_every=len(wl.ops) // 8, exact=exact)
    assert len(g) > 1000


def test_kicked_ising_clifford_angle_equals_cz_sdag():
    # RZZ(-pi/2) as Clifford == the reference's CZ, S_DAG, S_DAG composition
    rng = np.random.default_rng(3)
    n = 16
    words = ["".join(rng.choice(list("IXYZ"), n)) for _ in range(50)]
    terms = [(w, float(rng.uniform(-1, 1))) for w in dict.fromkeys(words)]
    bonds = C.lattice_bonds(4)
    g = gpu_from(terms, n, thr=0.0, clifford_angles=True)
    g.run([G.r2(G.RZZ, a, b, -math.pi / 2) for a, b in bonds])
    o = oracle_from(terms, n, thr=0.0)
    ops = []
    for a, b in bonds:
        ops += [G.g2(G.CZ, a, b), G.g1(G.S_DAG, a), G.g1(G.S_DAG, b)]
    o.run_ops(ops)
    same(g, o)


@pytest.mark.parametrize("exact", [True, False])
def test_clifford_t_prefix(exact):
    # the term count grows ~2-4x per layer past layer 15 (6480 terms after 16 layers)
    wl = C.clifford_t(layers=16)
    run_both(wl.observable, wl.n_qubits, wl.ops, thr=wl.min_abs_coeff, check_every=50, exact=exact)


@pytest.mark.parametrize("exact", [True, False])
def test_live_counts_match_oracle(exact):
    for wl in (C.tfim_1d(steps=3), C.kicked_ising_2d(layers=4)):
        g = gpu_from(wl.observable, wl.n_qubits, wl.min_abs_coeff, wl.max_weight, wl.clifford_angles, exact=exact)
        o = oracle_from(wl.observable, wl.n_qubits, wl.min_abs_coeff, wl.max_weight, wl.clifford_angles)
        g.run(wl.ops)
        want = o.run_ops(wl.ops, counts=True)
        assert np.array_equal(g.live_counts(), want)


def test_preserve_strings():
    n = 4
    single = [C._z_word(n, j) for j in range(n)]
    g = PauliSum(single, n, min_abs_coeff=0.5, preserve_strings=single)
    o = oracle_from([(w, 1.0) for w in single], n, thr=0.5)
    o.set_preserve(*planes(single, n))
    for a, b in ((0, 1), (1, 2), (2, 3)):
        ops = [G.r2(G.RXX, a, b, 0.37), G.r2(G.RYY, a, b, 0.37), G.truncate()]
        g.run(ops)
        o.run_ops(ops)
        same(g, o)
    g = PauliSum(["ZII", "IZI", "IIZ", "XYZ", "XXX"], 3, [1e-6, 1e-6, 1e-6, 1e-6, 0.7], min_abs_coeff=0.5,
                 preserve_strings=["ZII", "IZI", "IIZ"])
    g.truncate()
    assert [w for w, _ in g.terms] == ["XXX", "ZII", "IZI", "IIZ"]


def test_python_api_basics():
    # ppvm-python/test/test_basics.py
    s = PauliSum(n_qubits=2, initial_terms=["ZZ"], coefficients=[1.0])
    s.cnot(0, 1)
    s.h(0)
    assert str(s) == "1.000 * IZ"
    assert s.overlap_with_zero() == 1.0
    t = s.copy()
    assert t == s and len(t) == 1 and t.terms == [("IZ", 1.0)]
    n, w = 200, 80
    big = PauliSum([C._z_word(n, j) for j in range(n)], n, max_pauli_weight=w)
    for i in reversed(range(1, n)):
        big.cnot(i - 1, i)
    big.h(0)
    assert big.overlap_with_zero() == 0.0
    s = PauliSum(["IZ"], 2)
    assert s.current_max_weight() == 1
    s.cnot(0, 1)
    s.h(0)
    assert s.current_max_weight() == 2
    assert PauliSum(["ZX", "IY"], 2).weights() == [("ZX", 2), ("IY", 1)]
    with pytest.raises(ValueError):
        s.cnot(0, 1, 1)
    with pytest.raises(ValueError):
        s.rx(5, theta=0.1)


def test_truncate_kwarg_and_overlap_trace():
    a = PauliSum.new(3, "Z1", min_abs_coeff=1e-12)
    a.rxx(0, 1, theta=0.5, truncate=False)
    a.ryy(0, 1, theta=0.5, truncate=False)
    a.truncate()
    b = PauliSum.new(3, "Z1", min_abs_coeff=1e-12)
    b.rxx(0, 1, theta=0.5)
    b.ryy(0, 1, theta=0.5)
    assert dict(a.terms) == dict(b.terms)
    total = sum(a.overlap(PauliSum.new(3, f"Z{j}")) for j in range(3))
    assert abs(total - 1.0) < 1e-12
    s = PauliSum(["XYY", "ZIZ", "III", "IXI"], 3, [2.0, 3.0, 5.0, 7.0], min_abs_coeff=0.0)
    assert s.trace("Z?*") == 8.0
    assert s.trace("X0Y1Y2") == 2.0
    assert s.trace("[XY]*") == 7.0
    assert s.trace("X1") == 7.0


def test_empty_and_edge_cases():
    s = PauliSum(["XX"], 2, [1e-3], min_abs_coeff=0.5)
    s.truncate()
    assert len(s) == 0
    s.rx(0, 1, theta=0.3)
    s.h(0)
    assert len(s) == 0 and s.overlap_with_zero() == 0.0
    s = PauliSum(["ZZ"], 2, [1.0], min_abs_coeff=0.0)
    s.pauli_rotation("XY", 0.4)
    o = oracle_from([("ZZ", 1.0)], 2, thr=0.0)
    gx, gz = G.parse_word("XY", 2)
    o.pauli_rotation(gx, gz, 0.4)
    same(s, o)


def test_cached_buffers_are_reused_safely():
    # sums created after others were destroyed take their buffers from the cache: results
    # stay identical, also after the cache is handed back to the driver
    from ppvm_b200._lib import lib

    wl = C.kicked_ising_2d(layers=3)
    got = []
    for rep in range(3):
        g = gpu_from(wl.observable, wl.n_qubits, wl.min_abs_coeff, wl.max_weight, True, exact=False)
        g.run(wl.ops)
        got.append(_sorted(*g.export()))
        del g
        if rep == 1:
            assert lib().ppvm_release_cached_memory() == 0
    for k, c in got[1:]:
        assert np.array_equal(k, got[0][0]) and np.array_equal(c.view(np.uint64), got[0][1].view(np.uint64))


def test_reused_handles_start_clean():
    # a destroyed sum's handle is handed out again for the same width: nothing of the old sum
    # (terms, preserve strings, strategy, flags, counters) may leak into the new one
    a = PauliSum(["ZII", "XXX"], 3, [1e-6, 0.7], min_abs_coeff=0.5, preserve_strings=["ZII"], exact_order=True)
    a.truncate()
    assert [w for w, _ in a.terms] == ["XXX", "ZII"]
    del a
    for n in (3, 5):
        b = PauliSum(["Z" + "I" * (n - 1), "X" * n], n, [1e-6, 0.7], min_abs_coeff=0.5)
        assert len(b) == 2 and b.launch_count() < 10
        b.truncate()
        assert [w for w, _ in b.terms] == ["X" * n]
        del b
    wl = C.tfim_1d(steps=3)
    run_both(wl.observable, wl.n_qubits, wl.ops, thr=wl.min_abs_coeff, check_every=40, exact=False)


@pytest.mark.parametrize("n", [7, 64, 100, 144, 300])
def test_overlap_matches_oracle_on_random_sums(n):
    # PauliSum::overlap (crates/ppvm-pauli-sum/src/sum/trace.rs:31-37): sum over the other
    # sum's terms of its coefficient times this sum's coefficient of the same word.  Two
    # random sums sharing about a third of their words, both propagated a little first
    rng = np.random.default_rng(500 + n)

    def words(m):
        out = set()
        while len(out) < m:
            w = ["I"] * n
            for q in rng.choice(n, int(rng.integers(1, 6)), replace=False):
                w[int(q)] = "XYZ"[int(rng.integers(3))]
            out.add("".join(w))
        return sorted(out)

    shared, only_a, only_b = words(300), words(400), words(200)
    ta = [(w, float(rng.uniform(-1, 1))) for w in dict.fromkeys(shared + only_a)]
    tb = [(w, float(rng.uniform(-1, 1))) for w in dict.fromkeys(only_b + shared)]
    ops = [G.r1(G.RX, int(q), 0.2) for q in rng.choice(n, min(n, 5), replace=False)] + [G.truncate()]
    for exact in (True, False):
        ga, gb = gpu_from(ta, n, thr=1e-6, exact=exact), gpu_from(tb, n, thr=1e-6, exact=exact)
        oa, ob = oracle_from(ta, n, thr=1e-6), oracle_from(tb, n, thr=1e-6)
        for g, o in ((ga, oa), (gb, ob)):
            g.run(ops)
            o.run_ops(ops)
        want = oa.overlap(ob)
        assert abs(ga.overlap(gb) - want) < 1e-10, (ga.overlap(gb), want)
        assert abs(gb.overlap(ga) - ob.overlap(oa)) < 1e-10
        assert abs(ga.overlap(ga) - oa.overlap(oa)) < 1e-10
    disjoint = gpu_from([("Y" * n, 1.0)], n)
    assert ga.overlap(disjoint) == 0.0
