"""The composed Clifford map of a gate run (host side, no GPU).

The engine applies runs of 8 or more Clifford gates as one composed map: the images of the
generators X_q, Z_q (the Clifford tableau), composed on the host, and one product of images
per term on the device.  These tests check, against the oracle's gate-by-gate restatement of
the reference (crates/ppvm-pauli-sum/src/sum/clifford.rs:37-221), that

  * every image the host composes equals the oracle's propagation of that generator, and
  * the per-term product rule the device kernel uses (restated here in Python) maps random
    words exactly as the oracle does, sign included.
"""

import math
import random

import numpy as np
import pytest

from ppvm_b200 import gates as G
from ppvm_b200.paulisum import clifford_tableau
from tests.helpers import oracle_from

CLIFF1 = sorted(G.SINGLE_CLIFFORD)
CLIFF2 = sorted(G.TWO_CLIFFORD)


def random_clifford_ops(rng, n, L, angles=True):
    ops = []
    for _ in range(L):
        r = rng.random()
        if r < 0.45 or n == 1:
            ops.append(G.g1(rng.choice(CLIFF1), rng.randrange(n)))
        elif r < 0.8:
            a, b = rng.sample(range(n), 2)
            ops.append(G.g2(rng.choice(CLIFF2), a, b))
        elif angles and r < 0.9:
            ops.append(G.r1(rng.choice(sorted(G.ROT1)), rng.randrange(n), rng.choice([-1, 1]) * G.HALF_PI))
        elif angles:
            a, b = rng.sample(range(n), 2)
            ops.append(G.r2(rng.choice(sorted(G.ROT2)), a, b, rng.choice([-1, 1]) * G.HALF_PI))
        else:
            ops.append(G.g1(rng.choice(CLIFF1), rng.randrange(n)))
    return ops


def unit_word(n, q, kind):
    return "".join(("X" if kind == 0 else "Z") if i == q else "I" for i in range(n))


def oracle_image(n, word, ops):
    o = oracle_from([(word, 1.0)], n, thr=0.0, clifford_angles=True)
    o.run_ops(ops)
    x, z, c = o.export()
    assert len(c) == 1
    assert abs(c[0]) == 1.0
    return x[0], z[0], c[0]


def popc(a):
    return sum(bin(int(v)).count("1") for v in a)


def apply_tableau(ix, iz, sg, x, z):
    """The kernel's product rule: P = i^{|x&z|} X^x Z^z -> prod f(X_q) prod f(Z_q), images
    held as i^ph X^a Z^b, and X^u Z^v X^a Z^b = (-1)^{|v&a|} X^{u^a} Z^{v^b}."""
    W = len(x)
    n = ix.shape[0] // 2
    u = np.zeros(W, dtype=np.uint64)
    v = np.zeros(W, dtype=np.uint64)
    p = popc(x & z)
    for kind, plane in ((0, x), (1, z)):
        for q in range(n):
            if (int(plane[q // 64]) >> (q % 64)) & 1:
                row = 2 * q + kind
                a, b = ix[row], iz[row]
                ph = (popc(a & b) + 2 * int(sg[row])) & 3
                p += ph + 2 * popc(v & a)
                u ^= a
                v ^= b
    e = (p - popc(u & v)) & 3
    assert e in (0, 2), "image is not Hermitian"
    return u, v, (-1.0 if e == 2 else 1.0)


@pytest.mark.parametrize("n,L,seed", [(3, 40, 1), (7, 60, 2), (20, 120, 3), (70, 200, 4), (130, 150, 5)])
def test_generator_images_match_oracle(n, L, seed):
    rng = random.Random(seed)
    ops = random_clifford_ops(rng, n, L)
    ix, iz, sg = clifford_tableau(n, ops)
    for q in range(n):
        for kind in (0, 1):
            x, z, c = oracle_image(n, unit_word(n, q, kind), ops)
            row = 2 * q + kind
            assert np.array_equal(ix[row], x) and np.array_equal(iz[row], z), (q, kind)
            assert (c < 0) == bool(sg[row]), (q, kind)


@pytest.mark.parametrize("n,L,seed", [(5, 30, 11), (20, 100, 12), (64, 264, 13), (100, 80, 14)])
def test_product_rule_maps_random_words_like_the_oracle(n, L, seed):
    rng = random.Random(seed)
    ops = random_clifford_ops(rng, n, L)
    ix, iz, sg = clifford_tableau(n, ops)
    for _ in range(40):
        word = "".join(rng.choice("IXYZ") for _ in range(n))
        x0, z0 = G.parse_word(word, n)
        u, v, sign = apply_tableau(ix, iz, sg, x0, z0)
        x, z, c = oracle_image(n, word, ops)
        assert np.array_equal(u, x) and np.array_equal(v, z)
        assert sign == c


def test_kicked_ising_bond_layer_is_the_cz_sdag_layer():
    # RZZ(-pi/2) on every bond, as a Clifford angle, equals cz + s_dag on both qubits
    L = 4
    bonds = [(r * L + c, r * L + c + 1) for r in range(L) for c in range(L - 1)]
    bonds += [(r * L + c, (r + 1) * L + c) for r in range(L - 1) for c in range(L)]
    a = clifford_tableau(L * L, [G.r2(G.RZZ, p, q, -math.pi / 2) for p, q in bonds])
    ops = []
    for p, q in bonds:
        ops += [G.g2(G.CZ, p, q), G.g1(G.S_DAG, p), G.g1(G.S_DAG, q)]
    b = clifford_tableau(L * L, ops)
    for u, v in zip(a, b):
        assert np.array_equal(u, v)


def test_rejects_non_clifford_ops():
    with pytest.raises(ValueError):
        clifford_tableau(4, [G.r1(G.RX, 0, 0.3)])
    with pytest.raises(ValueError):
        clifford_tableau(4, [G.pauli_error(0, (0.1, 0.0, 0.0))])
    with pytest.raises(ValueError):
        clifford_tableau(4, [G.g1(G.H, 4)])


def chunk_tables(ix, iz, sg, n):
    """The one-word kernel's chunk tables: for each 4-qubit chunk c, the image of every
    sub-word X^{x_c} Z^{z_c} (index x nibble | z nibble << 4) as (a, b, ph), image =
    i^ph X^a Z^b, built per x nibble by a Gray-code walk over the z nibbles."""
    def gen(q, kind):
        if q >= n:  # beyond the register: the generator itself
            return (1 << q, 0, 0) if kind == 0 else (0, 1 << q, 0)
        row = 2 * q + kind
        a, b = int(ix[row][0]), int(iz[row][0])
        return a, b, (bin(a & b).count("1") + 2 * int(sg[row])) & 3

    def mul(acc, img):
        u, v, p = acc
        a, b, e = img
        return u ^ a, v ^ b, (p + e + 2 * bin(v & a).count("1")) & 3

    tab = {}
    for c in range(16):
        for xv in range(16):
            acc = (0, 0, 0)
            for j in range(4):
                if (xv >> j) & 1:
                    acc = mul(acc, gen(4 * c + j, 0))
            tab[c, xv] = acc
            g = 0
            for k in range(1, 16):
                j = (k & -k).bit_length() - 1
                g ^= 1 << j
                acc = mul(acc, gen(4 * c + j, 1))
                tab[c, xv | (g << 4)] = acc
    return tab


def apply_chunk_tables(tab, x, z):
    x, z = int(x[0]), int(z[0])
    u = v = 0
    p = bin(x & z).count("1")
    for c in range(16):
        a, b, e = tab[c, ((x >> (4 * c)) & 15) | (((z >> (4 * c)) & 15) << 4)]
        p += e + 2 * bin(v & a).count("1")
        u ^= a
        v ^= b
    e = (p - bin(u & v).count("1")) & 3
    assert e in (0, 2), "image is not Hermitian"
    return u, v, (-1.0 if e == 2 else 1.0)


@pytest.mark.parametrize("n,L,seed", [(1, 12, 24), (2, 20, 25), (5, 40, 21), (37, 150, 22), (64, 300, 23)])
def test_chunk_tables_map_words_like_the_oracle(n, L, seed):
    rng = random.Random(seed)
    ops = random_clifford_ops(rng, n, L)
    ix, iz, sg = clifford_tableau(n, ops)
    tab = chunk_tables(ix, iz, sg, n)
    for i in range(30):
        word = "".join(rng.choice("IXYZ" if i % 2 else "IIIIIIIXYZ") for _ in range(n))
        x0, z0 = G.parse_word(word, n)
        u, v, sign = apply_chunk_tables(tab, x0, z0)
        x, z, c = oracle_image(n, word, ops)
        assert u == int(x[0]) and v == int(z[0])
        assert sign == c
