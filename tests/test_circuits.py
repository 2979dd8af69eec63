"""Workload generators: shapes, counts and determinism (no GPU)."""

import hashlib
import math

from ppvm_b200 import circuits as C
from ppvm_b200 import gates as G


def _digest(ops):
    h = hashlib.sha256()
    for op in ops:
        h.update(repr((op[0], op[1], op[2], round(op[3], 15))).encode())
    return h.hexdigest()


def test_tfim_shape():
    wl = C.tfim_1d()
    assert wl.n_qubits == 20 and wl.n_gates == 10 * (19 + 20)
    assert wl.observable == [("I" * 10 + "Z" + "I" * 9, 1.0)]
    assert sum(op[0] == G.TRUNCATE for op in wl.ops) == 20
    assert wl.ops[0] == G.r1(G.RX, 19, 0.2)


def test_kicked_ising_shape():
    wl = C.kicked_ising_2d()
    assert wl.n_qubits == 144 and wl.meta["bonds"] == 264
    assert wl.n_gates == 20 * (144 + 264) and wl.clifford_angles
    assert wl.observable[0][0][78] == "Z"
    assert wl.ops[0] == G.r2(G.RZZ, 131, 143, -math.pi / 2)


def test_clifford_t_deterministic():
    a, b = C.clifford_t(layers=50), C.clifford_t(layers=50)
    assert _digest(a.ops) == _digest(b.ops)
    assert sum(ch != "I" for ch in a.observable[0][0]) == 4
    assert a.meta["t_gates"] > 0


def test_batched_ranges():
    wls = C.batched_tfim(count=64)
    assert len(wls) == 64
    assert all(16 <= w.n_qubits <= 128 and 5 <= w.meta["steps"] <= 30 for w in wls)
    assert all(0.5 <= w.meta["h"] <= 1.5 for w in wls)


def test_kicked_ising_observable_is_on_the_lattice():
    import pytest

    assert C.kicked_ising_2d(L=4, layers=1).observable[0][0] == "".join("Z" if q == 10 else "I" for q in range(16))
    assert C.kicked_ising_2d().observable[0][0].index("Z") == 6 * 12 + 6
    with pytest.raises(ValueError):
        C.kicked_ising_2d(L=4, layers=1, obs=(6, 6))
