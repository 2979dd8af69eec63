"""Gate-list encoding shared by the host API, the workload generators and the tests.

The opcodes mirror ``ppvm_opcode`` in include/ppvm_cuda.h.  A gate is a tuple
``(code, q0, q1, theta, (p0, p1, p2))``; helpers below build them.

Pauli words are held as two bit planes of ``W = ceil(n/64)`` u64 words, qubit ``q`` at
bit ``q % 64`` of word ``q // 64`` (the Lsb0 layout of ``PauliWord``,
crates/ppvm-pauli-word/src/word/data.rs:43-52 in the reference).
"""

from __future__ import annotations

import math

import numpy as np

X, Y, Z, H, S, S_DAG, SQRT_X, SQRT_X_DAG, SQRT_Y, SQRT_Y_DAG = range(10)
CNOT, CZ, CY = 10, 11, 12
RX, RY, RZ = 13, 14, 15
RXX, RYY, RZZ = 16, 17, 18
PAULI_ERROR, DEPOLARIZE1, DEPOLARIZE2 = 19, 20, 21
TRUNCATE = 22
AMPLITUDE_DAMPING = 23
LOSS_CHANNEL, RESET_LOSS_CHANNEL, CORRELATED_LOSS_CHANNEL = 24, 25, 26

NAMES = {
    X: "x", Y: "y", Z: "z", H: "h", S: "s", S_DAG: "s_dag", SQRT_X: "sqrt_x",
    SQRT_X_DAG: "sqrt_x_dag", SQRT_Y: "sqrt_y", SQRT_Y_DAG: "sqrt_y_dag", CNOT: "cnot",
    CZ: "cz", CY: "cy", RX: "rx", RY: "ry", RZ: "rz", RXX: "rxx", RYY: "ryy", RZZ: "rzz",
    PAULI_ERROR: "pauli_error", DEPOLARIZE1: "depolarize1", DEPOLARIZE2: "depolarize2",
    TRUNCATE: "truncate", AMPLITUDE_DAMPING: "amplitude_damping", LOSS_CHANNEL: "loss_channel",
    RESET_LOSS_CHANNEL: "reset_loss_channel", CORRELATED_LOSS_CHANNEL: "correlated_loss_channel",
}
SINGLE_CLIFFORD = {X, Y, Z, H, S, S_DAG, SQRT_X, SQRT_X_DAG, SQRT_Y, SQRT_Y_DAG}
TWO_CLIFFORD = {CNOT, CZ, CY}
ROT1 = {RX, RY, RZ}
ROT2 = {RXX, RYY, RZZ}
HALF_PI = math.pi / 2

_ZERO3 = (0.0, 0.0, 0.0)


def g1(code: int, q: int):
    return (code, q, 0, 0.0, _ZERO3)


def g2(code: int, a: int, b: int):
    return (code, a, b, 0.0, _ZERO3)


def r1(code: int, q: int, theta: float):
    return (code, q, 0, float(theta), _ZERO3)


def r2(code: int, a: int, b: int, theta: float):
    return (code, a, b, float(theta), _ZERO3)


def pauli_error(q: int, p):
    return (PAULI_ERROR, q, 0, 0.0, tuple(float(v) for v in p))


def depolarize1(q: int, p: float):
    return (DEPOLARIZE1, q, 0, float(p), _ZERO3)


def depolarize2(a: int, b: int, p: float):
    return (DEPOLARIZE2, a, b, float(p), _ZERO3)


def amplitude_damping(q: int, gamma: float):
    return (AMPLITUDE_DAMPING, q, 0, float(gamma), _ZERO3)


def loss_channel(q: int, p: float):
    return (LOSS_CHANNEL, q, 0, float(p), _ZERO3)


def reset_loss_channel(q: int):
    return (RESET_LOSS_CHANNEL, q, 0, 0.0, _ZERO3)


def correlated_loss_channel(a: int, b: int, p):
    return (CORRELATED_LOSS_CHANNEL, a, b, 0.0, tuple(float(v) for v in p))


def truncate():
    return (TRUNCATE, 0, 0, 0.0, _ZERO3)


def words(n_qubits: int) -> int:
    return (n_qubits + 63) // 64


_XBITS = str.maketrans("IXYZ", "0110")
_ZBITS = str.maketrans("IXYZ", "0011")
_M64 = (1 << 64) - 1


def parse_word(s: str, n_qubits: int | None = None):
    """Pauli string -> (x[W], z[W]) u64 planes; '_' is skipped like the reference parser
    (crates/ppvm-pauli-word/src/word/data.rs:332-377)."""
    t = s.replace("_", "")
    n = len(t) if n_qubits is None else n_qubits
    if len(t) != n:
        raise ValueError(f"word {s!r} has {len(t)} qubits, expected {n}")
    if t.strip("IXYZ"):  # non-empty exactly when some character is not a Pauli letter
        bad = next(c for c in t if c not in "IXYZ")
        raise ValueError(f"Invalid Pauli character: {bad}")
    W = words(n)
    # character q is bit q: reversed, the 0/1 string reads as a binary number
    xv = int(t.translate(_XBITS)[::-1] or "0", 2)
    zv = int(t.translate(_ZBITS)[::-1] or "0", 2)
    x = np.array([(xv >> (64 * w)) & _M64 for w in range(W)], dtype=np.uint64)
    z = np.array([(zv >> (64 * w)) & _M64 for w in range(W)], dtype=np.uint64)
    return x, z


def lossy_words(n_qubits: int) -> int:
    """Words per plane of a lossy sum: the X plane's upper half holds the loss bits."""
    return 2 * words(n_qubits)


def parse_lossy_word(s: str, n_qubits: int | None = None):
    """Lossy Pauli string (I, X, Y, Z, L) -> (x[2W], z[2W]) in the lossy layout: loss bit of
    qubit q at bit q % 64 of X word W + q // 64 (crates/ppvm-pauli-word/src/loss/data.rs:318-377
    parses the same alphabet; '_' is skipped)."""
    chars = [c for c in s if c != "_"]
    n = len(chars) if n_qubits is None else n_qubits
    if len(chars) != n:
        raise ValueError(f"word {s!r} has {len(chars)} qubits, expected {n}")
    W = words(n)
    x = np.zeros(2 * W, dtype=np.uint64)
    z = np.zeros(2 * W, dtype=np.uint64)
    plain = "".join("I" if c == "L" else c for c in chars)
    x[:W], z[:W] = parse_word(plain, n)
    for q, c in enumerate(chars):
        if c == "L":
            x[W + q // 64] |= np.uint64(1) << np.uint64(q % 64)
    return x, z


def lossy_word_str(x, z, n_qubits: int) -> str:
    W = words(n_qubits)
    out = list(word_str(x[:W], z[:W], n_qubits))
    for q in range(n_qubits):
        if (int(x[W + q // 64]) >> (q % 64)) & 1:
            out[q] = "L"
    return "".join(out)


def word_str(x, z, n_qubits: int) -> str:
    out = []
    for q in range(n_qubits):
        xb = (int(x[q // 64]) >> (q % 64)) & 1
        zb = (int(z[q // 64]) >> (q % 64)) & 1
        out.append("IXZY"[xb | (zb << 1)])
    return "".join(out)


def weight(x, z) -> int:
    return int(sum(bin(int(a) | int(b)).count("1") for a, b in zip(x, z)))


def reverse_heisenberg(forward):
    """Heisenberg order is the exact reverse of the forward gate list."""
    return list(reversed(forward))
