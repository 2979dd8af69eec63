"""Independent check of the oracle's Heisenberg propagation against a numpy state vector.

For random circuits on n <= 6 qubits, <0|U^dag O U|0> from the state vector must equal the
oracle's overlap_with_zero after propagating O through the reversed circuit, untruncated,
to 1e-9 (the idea of ppvm-python/test/test_heisenberg_ordering.py:74-203).
"""

import math

import numpy as np
import pytest

from ppvm_b200 import gates as G
from tests.helpers import oracle_from

I2 = np.eye(2, dtype=complex)
PX = np.array([[0, 1], [1, 0]], dtype=complex)
PY = np.array([[0, -1j], [1j, 0]], dtype=complex)
PZ = np.array([[1, 0], [0, -1]], dtype=complex)
PAULI = {"I": I2, "X": PX, "Y": PY, "Z": PZ}


def rot(P, t):
    return math.cos(t / 2) * I2 - 1j * math.sin(t / 2) * P


ONE_Q = {
    G.X: PX, G.Y: PY, G.Z: PZ, G.H: np.array([[1, 1], [1, -1]], dtype=complex) / math.sqrt(2),
    G.S: np.diag([1, 1j]), G.S_DAG: np.diag([1, -1j]),
    G.SQRT_X: rot(PX, math.pi / 2), G.SQRT_X_DAG: rot(PX, -math.pi / 2),
    G.SQRT_Y: rot(PY, math.pi / 2), G.SQRT_Y_DAG: rot(PY, -math.pi / 2),
}


def apply1(psi, U, q, n):
    psi = psi.reshape([2] * n)
    psi = np.moveaxis(np.tensordot(U, psi, axes=([1], [q])), 0, q)
    return psi.reshape(-1)


def apply2(psi, U4, a, b, n):
    psi = psi.reshape([2] * n)
    U = U4.reshape(2, 2, 2, 2)
    psi = np.tensordot(U, psi, axes=([2, 3], [a, b]))
    psi = np.moveaxis(psi, [0, 1], [a, b])
    return psi.reshape(-1)


def two_q(code, theta):
    if code == G.CNOT:
        return np.array([[1, 0, 0, 0], [0, 1, 0, 0], [0, 0, 0, 1], [0, 0, 1, 0]], dtype=complex)
    if code == G.CZ:
        return np.diag([1, 1, 1, -1]).astype(complex)
    if code == G.CY:
        m = np.eye(4, dtype=complex)
        m[2:, 2:] = PY
        return m
    P = {G.RXX: PX, G.RYY: PY, G.RZZ: PZ}[code]
    PP = np.kron(P, P)
    return math.cos(theta / 2) * np.eye(4) - 1j * math.sin(theta / 2) * PP


def observable(word):
    # qubit 0 is the most significant tensor factor in the reshape([2]*n) convention
    m = np.array([[1.0]], dtype=complex)
    for ch in word:
        m = np.kron(m, PAULI[ch])
    return m


@pytest.mark.parametrize("seed", range(12))
def test_random_circuit_matches_statevector(seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(2, 7))
    ops = []
    for _ in range(int(rng.integers(5, 25))):
        kind = rng.integers(0, 4)
        if kind == 0:
            ops.append(G.g1(int(rng.choice(sorted(ONE_Q))), int(rng.integers(n))))
        elif kind == 1:
            ops.append(G.r1(int(rng.choice([G.RX, G.RY, G.RZ])), int(rng.integers(n)), float(rng.uniform(-3, 3))))
        else:
            a, b = (int(v) for v in rng.choice(n, 2, replace=False))
            code = int(rng.choice([G.CNOT, G.CZ, G.CY, G.RXX, G.RYY, G.RZZ]))
            ops.append(G.r2(code, a, b, float(rng.uniform(-3, 3))) if code in G.ROT2 else G.g2(code, a, b))
    word = "".join(rng.choice(list("IXYZ")) for _ in range(n))
    psi = np.zeros(2 ** n, dtype=complex)
    psi[0] = 1.0
    for code, q0, q1, th, _ in ops:
        if code in ONE_Q:
            psi = apply1(psi, ONE_Q[code], q0, n)
        elif code in G.ROT1:
            P = {G.RX: PX, G.RY: PY, G.RZ: PZ}[code]
            psi = apply1(psi, rot(P, th), q0, n)
        else:
            psi = apply2(psi, two_q(code, th), q0, q1, n)
    want = float(np.real(np.vdot(psi, observable(word) @ psi)))
    s = oracle_from([(word, 1.0)], n, thr=0.0)
    s.run_ops(G.reverse_heisenberg(ops))
    assert abs(s.overlap_with_zero() - want) < 1e-9
