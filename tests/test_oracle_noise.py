"""The oracle's two-qubit Pauli error and amplitude damping.

Three kinds of check:
- the reference's own known answers (crates/ppvm-pauli-sum/tests/noise.rs:8-95 and 223-265);
- every factor of the two-qubit channel against 1 - 2 * (sum of p over the anticommuting
  Paulis), computed here from the symplectic product;
- an independent numpy density-matrix evolution with the channels' Kraus operators.
"""

import itertools
import math

import numpy as np
import pytest

from ppvm_b200 import gates as G
from tests.helpers import oracle_dict, oracle_from
from tests.test_oracle_statevector import ONE_Q, PAULI, apply1, observable, rot, two_q

ORDER = ["IX", "IY", "IZ", "XI", "XX", "XY", "XZ", "YI", "YX", "YY", "YZ", "ZI", "ZX", "ZY", "ZZ"]
SYMP = {"I": (0, 0), "X": (1, 0), "Z": (0, 1), "Y": (1, 1)}


def anticommute(a: str, b: str) -> bool:
    s = 0
    for pa, pb in zip(a, b):
        xa, za = SYMP[pa]
        xb, zb = SYMP[pb]
        s ^= (xa & zb) ^ (za & xb)
    return bool(s)


def perr2(s, a, b, p, truncate=False):
    s.two_qubit_pauli_error([a, b], p, truncate=truncate)


def test_two_qubit_pauli_error_known_answers():
    # tests/noise.rs:8-95: one unit probability at a time is the matching Pauli gate
    p = [0.0] * 15
    s = oracle_from([("IZ", 1.0)], 2)
    p[0] = 1.0  # IX
    perr2(s, 0, 1, p)
    assert oracle_dict(s) == {"IZ": -1.0}  # = x(1)
    p[0], p[1] = 0.0, 1.0  # IY
    perr2(s, 0, 1, p)
    assert oracle_dict(s) == {"IZ": 1.0}  # = y(1) again
    s = oracle_from([("IX", 1.0)], 2)
    p[1], p[2] = 0.0, 1.0  # IZ
    perr2(s, 0, 1, p)
    assert oracle_dict(s) == {"IX": -1.0}
    p[2] = 0.0
    s = oracle_from([("YI", 1.0)], 2)
    p[4] = 1.0  # XX on YI: rxx(pi) then truncate
    perr2(s, 0, 1, p)
    assert oracle_dict(s) == {"YI": -1.0}
    s = oracle_from([("YZ", 1.0)], 2)
    perr2(s, 0, 1, p)  # XX commutes with YZ
    assert oracle_dict(s) == {"YZ": 1.0}
    p[4] = 0.0
    s = oracle_from([("XI", 1.0)], 2)
    p[14] = 1.0  # ZZ
    perr2(s, 0, 1, p)
    assert oracle_dict(s) == {"XI": -1.0}
    s = oracle_from([("XI", 1.0)], 2)
    p[4] = 1.0  # XX and ZZ together: 1 - 2 * 1 (only ZZ anticommutes with XI)
    perr2(s, 0, 1, p)
    assert oracle_dict(s) == {"XI": -1.0}


@pytest.mark.parametrize("seed", range(4))
def test_two_qubit_pauli_error_factors(seed):
    rng = np.random.default_rng(seed)
    p = rng.uniform(0, 1 / 15, 15)
    for pa, pb in itertools.product("IXYZ", repeat=2):
        word = pa + "I" + pb  # the pair is (0, 2), qubit 1 untouched
        s = oracle_from([(word, 1.0)], 3)
        s.two_qubit_pauli_error([0, 2], p, truncate=False)
        got = oracle_dict(s)[word]
        want = 1.0 - 2.0 * sum(p[i] for i, q in enumerate(ORDER) if anticommute(pa + pb, q))
        assert abs(got - want) < 1e-15, (pa, pb, got, want)
    s = oracle_from([("XYZ", 0.5)], 3)
    with pytest.raises(ValueError):
        s.two_qubit_pauli_error([0, 1, 2], p)  # odd pair list
    with pytest.raises(ValueError):
        s.two_qubit_pauli_error([1, 1], p)  # repeated qubit


def test_amplitude_damping_known_answers():
    # tests/noise.rs:223-265
    g = 0.3
    s = oracle_from([("ZI", 1.0)], 2)
    s.run_ops([G.amplitude_damping(0, g)])
    d = oracle_dict(s)
    assert abs(d["ZI"] - (1.0 - g)) < 1e-10 and abs(d["II"] - g) < 1e-10
    s = oracle_from([("XI", 1.0)], 2)
    s.run_ops([G.amplitude_damping(0, g)])
    x = oracle_dict(s)["XI"]
    assert abs(x - math.sqrt(1.0 - g)) < 1e-10
    assert abs(x * x - (1.0 - g)) < 1e-10
    s = oracle_from([("II", 1.0)], 2)
    s.run_ops([G.amplitude_damping(0, g)])
    assert oracle_dict(s) == {"II": 1.0}


def test_amplitude_damping_merges_and_appends_in_parent_order():
    # map_insert: parents scaled in place, each child (Z -> I on q) merged with `+=` into an
    # existing term or appended after all terms, in parent order
    g = 0.25
    s = oracle_from([("ZX", 0.5), ("IX", 0.125), ("ZZ", -1.0), ("YI", 2.0), ("ZY", 0.75)], 2)
    s.run_ops([G.amplitude_damping(0, g)])
    x, z, c = s.export()
    words = [G.word_str(x[i], z[i], 2) for i in range(len(c))]
    assert words == ["ZX", "IX", "ZZ", "YI", "ZY", "IZ", "IY"]
    assert c[1] == 0.125 + 0.5 * g  # merged child
    assert c[0] == 0.5 * (1.0 - g) and c[3] == 2.0 * math.sqrt(1.0 - g)
    assert c[5] == -1.0 * g and c[6] == 0.75 * g


# ---- density-matrix check ----------------------------------------------------------------
def dm_apply1(rho, U, q, n):
    rho = rho.reshape([2] * (2 * n))
    rho = np.moveaxis(np.tensordot(U, rho, axes=([1], [q])), 0, q)
    rho = np.moveaxis(np.tensordot(rho, U.conj().T, axes=([n + q], [0])), -1, n + q)
    return rho.reshape(2 ** n, 2 ** n)


def dm_unitary(rho, op, n):
    code, q0, q1, th, _ = op
    if code in ONE_Q:
        return dm_apply1(rho, ONE_Q[code], q0, n)
    if code in G.ROT1:
        return dm_apply1(rho, rot({G.RX: PAULI["X"], G.RY: PAULI["Y"], G.RZ: PAULI["Z"]}[code], th), q0, n)
    U = two_q(code, th)
    full = embed2(U, q0, q1, n)
    return full @ rho @ full.conj().T


def embed2(U4, a, b, n):
    m = np.zeros((2 ** n, 2 ** n), dtype=complex)
    for col in range(2 ** n):
        e = np.zeros(2 ** n, dtype=complex)
        e[col] = 1.0
        psi = e.reshape([2] * n)
        psi = np.tensordot(U4.reshape(2, 2, 2, 2), psi, axes=([2, 3], [a, b]))
        psi = np.moveaxis(psi, [0, 1], [a, b])
        m[:, col] = psi.reshape(-1)
    return m


def pauli_on(word_pair, a, b, n):
    w = ["I"] * n
    w[a], w[b] = word_pair[0], word_pair[1]
    return observable("".join(w))


def dm_damp(rho, q, g, n):
    k0 = np.array([[1, 0], [0, math.sqrt(1 - g)]], dtype=complex)
    k1 = np.array([[0, math.sqrt(g)], [0, 0]], dtype=complex)
    return dm_apply1(rho, k0, q, n) + dm_apply1(rho, k1, q, n)


@pytest.mark.parametrize("seed", range(10))
def test_channels_match_density_matrix(seed):
    rng = np.random.default_rng(1000 + seed)
    n = int(rng.integers(2, 5))
    items = []
    for _ in range(int(rng.integers(6, 18))):
        kind = int(rng.integers(0, 5))
        if kind == 0:
            items.append(("op", G.g1(int(rng.choice(sorted(ONE_Q))), int(rng.integers(n)))))
        elif kind == 1:
            items.append(("op", G.r1(int(rng.choice([G.RX, G.RY, G.RZ])), int(rng.integers(n)),
                                     float(rng.uniform(-3, 3)))))
        elif kind == 2:
            a, b = (int(v) for v in rng.choice(n, 2, replace=False))
            items.append(("op", G.g2(int(rng.choice([G.CNOT, G.CZ])), a, b)))
        elif kind == 3:
            items.append(("op", G.amplitude_damping(int(rng.integers(n)), float(rng.uniform(0, 1)))))
        else:
            a, b = (int(v) for v in rng.choice(n, 2, replace=False))
            items.append(("perr2", a, b, rng.uniform(0, 1 / 15, 15)))
    rho = np.zeros((2 ** n, 2 ** n), dtype=complex)
    rho[0, 0] = 1.0
    for it in items:
        if it[0] == "op":
            op = it[1]
            rho = dm_damp(rho, op[1], op[3], n) if op[0] == G.AMPLITUDE_DAMPING else dm_unitary(rho, op, n)
        else:
            _, a, b, p = it
            new = (1.0 - p.sum()) * rho
            for i, q in enumerate(ORDER):
                P = pauli_on(q, a, b, n)
                new = new + p[i] * (P @ rho @ P)
            rho = new
    word = "".join(rng.choice(list("IXYZ")) for _ in range(n))
    want = float(np.real(np.trace(observable(word) @ rho)))
    s = oracle_from([(word, 1.0)], n, thr=0.0)
    chunk = []
    for it in reversed(items):
        if it[0] == "op":
            chunk.append(it[1])
        else:
            if chunk:
                s.run_ops(chunk)
                chunk = []
            s.two_qubit_pauli_error([it[1], it[2]], it[3], truncate=False)
    if chunk:
        s.run_ops(chunk)
    assert abs(s.overlap_with_zero() - want) < 1e-9
