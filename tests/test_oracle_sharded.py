"""The oracle's restatement of the reference's DashMap configuration (the one bench.py's
reference arm times on every host core) against its IndexMap configuration (the one the
parity tests use).  Both are the reference's PauliSum over different maps, so they hold the
same terms with every coefficient equal bit for bit (a key takes at most two contributions
per gate, so the merge order cannot change a sum); only the term order differs.  Traces sum
in a different order, so they are compared to 1e-12.  Runs on the CPU."""

import numpy as np
import pytest

from oracle.pyoracle import OracleSum
from ppvm_b200 import circuits as C
from ppvm_b200 import gates as G
from tests.helpers import planes
from tests.test_gpu_parity import random_case


def both(terms, n, thr=1e-10, maxw=None, clifford_angles=False, threads=3):
    a = OracleSum(n, thr, maxw, clifford_angles)
    b = OracleSum(n, thr, maxw, clifford_angles, threads=threads)
    if terms:
        x, z = planes([t for t, _ in terms], n)
        c = np.array([v for _, v in terms], dtype=np.float64)
        a.add_terms(x, z, c)
        b.add_terms(x, z, c)
    return a, b


def sorted_terms(o):
    x, z, c = o.export()
    keys = np.concatenate([x, z, c.view(np.uint64)[:, None]], axis=1)
    return keys[np.lexsort(keys.T[::-1])] if len(c) else keys


def check(a, b):
    assert len(a) == len(b)
    assert np.array_equal(sorted_terms(a), sorted_terms(b))
    assert abs(a.overlap_with_zero() - b.overlap_with_zero()) < 1e-12


@pytest.mark.parametrize("threads", [1, 4])
@pytest.mark.parametrize("n", [5, 64, 65, 144, 200])
def test_random_circuits(n, threads):
    terms, ops = random_case(n, n)
    a, b = both(terms, n, thr=1e-4, maxw=8, threads=threads)
    for i in range(0, len(ops), 40):
        ca = a.run_ops(ops[i:i + 40], counts=True)
        cb = b.run_ops(ops[i:i + 40], counts=True)
        assert np.array_equal(ca, cb)
        check(a, b)


def test_kicked_ising_prefix_and_noise():
    wl = C.kicked_ising_2d(layers=3)
    a, b = both(wl.observable, wl.n_qubits, wl.min_abs_coeff, wl.max_weight, True, threads=8)
    assert np.array_equal(a.run_ops(wl.ops, counts=True), b.run_ops(wl.ops, counts=True))
    check(a, b)
    ops = [G.depolarize1(5, 0.01), G.depolarize2(5, 6, 0.02), G.pauli_error(7, (0.01, 0.02, 0.03)),
           G.amplitude_damping(78, 0.1), G.truncate()]
    a.run_ops(ops)
    b.run_ops(ops)
    check(a, b)
    for pat in ("Z?*", "[XY]*", "Z78"):
        assert abs(a.trace(pat) - b.trace(pat)) < 1e-12


def test_preserve_strings_overlap_and_clone():
    n = 4
    single = [C._z_word(n, j) for j in range(n)]
    a, b = both([(w, 1.0) for w in single], n, thr=0.5)
    for o in (a, b):
        o.set_preserve(*planes(single, n))
    for p, q in ((0, 1), (1, 2), (2, 3)):
        ops = [G.r2(G.RXX, p, q, 0.37), G.r2(G.RYY, p, q, 0.37), G.truncate()]
        a.run_ops(ops)
        b.run_ops(ops)
        check(a, b)
    bc = b.clone()
    bc.run_ops([G.r1(G.RX, 0, 0.2)])
    a2 = a.clone()
    a2.run_ops([G.r1(G.RX, 0, 0.2)])
    check(a2, bc)
    assert abs(a.overlap(a2) - b.overlap(bc)) < 1e-12
