"""Pins the oracle's lossy words (LossyPauliWord) to the reference's own loss tests.

Each case restates a test of the reference (file:line cited): the lossy Clifford tables of
crates/ppvm-pauli-word/src/loss/clifford.rs (read into tests/golden/reference_tables.json by
make_golden.py) and the channel and gate cases of crates/ppvm-pauli-sum/tests/loss.rs.
``assert_eq!`` on two sums compares them as maps (IndexMap equality ignores order), so the
cases here compare term dicts.  These run without a GPU.
"""

import json
import os

import numpy as np
import pytest

from ppvm_b200 import gates as G
from tests.helpers import lossy_dict, lossy_list, lossy_oracle_from, lossy_planes, oracle_from

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_tables.json")))
OPS = {"x": G.X, "y": G.Y, "z": G.Z, "h": G.H, "s": G.S, "s_dag": G.S_DAG, "sqrt_x": G.SQRT_X,
       "sqrt_x_dag": G.SQRT_X_DAG, "sqrt_y": G.SQRT_Y, "sqrt_y_dag": G.SQRT_Y_DAG, "cnot": G.CNOT,
       "cz": G.CZ, "cy": G.CY}


@pytest.mark.parametrize("name", sorted(GOLD["loss_word_tables"]))
def test_lossy_clifford_tables(name):
    # crates/ppvm-pauli-word/src/loss/clifford.rs:13-207: gates on a lost qubit leave the word alone
    for inp, out in GOLD["loss_word_tables"][name]:
        n = len(inp)
        s = lossy_oracle_from([(inp, 1.0)], n)
        s.run_ops([G.g1(OPS[name], 0)] if n == 1 else [G.g2(OPS[name], 0, 1)])
        assert list(lossy_dict(s)) == [out], (name, inp)


def run(terms, n, ops, **kw):
    s = lossy_oracle_from(terms, n, **kw)
    s.run_ops(ops)
    return s


def test_lossy_sum():  # tests/loss.rs:14-25
    assert len(lossy_oracle_from([("ZI", 1.0), ("IZ", 1.0), ("LL", 1.0)], 2)) == 3


def test_reset_channel():  # tests/loss.rs:27-70
    assert lossy_dict(run([("X", 1.0)], 1, [G.reset_loss_channel(0)])) == {"X": 1.0}
    assert lossy_dict(run([("Y", 1.0)], 1, [G.reset_loss_channel(0)])) == {"Y": 1.0}
    assert lossy_dict(run([("I", 1.0)], 1, [G.reset_loss_channel(0)])) == {"I": 1.0, "L": 1.0}
    assert lossy_dict(run([("Z", 1.0)], 1, [G.reset_loss_channel(0)])) == {"Z": 1.0, "L": 1.0}
    assert lossy_dict(run([("L", 1.0)], 1, [G.reset_loss_channel(0)])) == {"L": 0.0}


def test_loss_channel():  # tests/loss.rs:72-115
    for w in "XYIZ":
        assert lossy_dict(run([(w, 1.0)], 1, [G.loss_channel(0, 0.2)])) == {w: 1.0 * 0.8}
    assert lossy_dict(run([("L", 1.0)], 1, [G.loss_channel(0, 0.2)])) == {"L": 1.0, "I": 0.2}


def test_single_qubit_loss():  # tests/loss.rs:117-141
    s = run([("Z", 1.0)], 1, [G.reset_loss_channel(0)])
    mid = lossy_dict(s)
    s.run_ops([G.g1(G.X, 0), G.g1(G.X, 0)])
    assert lossy_dict(s) == mid
    s.run_ops([G.loss_channel(0, 0.1), G.g1(G.X, 0)])
    assert abs(s.trace("Z?*") + 0.8) < 1e-10
    assert s.trace("Z?*") == s.overlap_with_zero()


def test_ghz_final_loss():  # tests/loss.rs:143-177
    p_l = 0.1
    ops = [G.reset_loss_channel(0), G.reset_loss_channel(1), G.g1(G.X, 0), G.g1(G.X, 1), G.g1(G.X, 0),
           G.g1(G.X, 1), G.loss_channel(0, p_l), G.loss_channel(1, p_l), G.g2(G.CNOT, 0, 1), G.g1(G.H, 0)]
    s = run([("ZZ", 1.0)], 2, ops)
    prob = 0.5 + 0.5 * ((1.0 - p_l) * (1.0 - p_l) - 2.0 * p_l * (1.0 - p_l) + p_l * p_l)
    assert abs(s.trace("Z?*") - prob) < 1e-10


def test_ghz():  # tests/loss.rs:179-207
    p_l = 0.1
    ops = [G.reset_loss_channel(0), G.reset_loss_channel(1), G.loss_channel(0, p_l), G.loss_channel(1, p_l),
           G.g2(G.CNOT, 0, 1), G.loss_channel(0, 2.0 * p_l), G.g1(G.H, 0)]
    s = run([("ZZ", 1.0)], 2, ops)
    prob = 2.0 * p_l + (1.0 - 2.0 * p_l) * (0.5 + 0.5 * ((1.0 - p_l) * (1.0 - p_l) - 2.0 * p_l * (1.0 - p_l)
                                                          + p_l * p_l))
    assert abs(s.trace("Z?*") - prob) < 1e-10


def test_loss_truncation():  # tests/loss.rs:209-241: MaxLossWeight(2) drops the LLL term
    ops = [G.reset_loss_channel(q) for q in range(3)] + [G.loss_channel(q, 0.1) for q in range(3)]
    s = run([("ZZZ", 1.0)], 3, ops, max_loss_weight=2)
    before = len(s)
    s.run_ops([G.truncate()])
    assert len(s) == before - 1 and "LLL" not in lossy_dict(s)


def test_reset_loss_channel_accumulates_duplicate_target():  # tests/loss.rs:243-277
    s = run([("I", 2.0), ("Z", 3.0)], 1, [G.reset_loss_channel(0)])
    assert lossy_dict(s) == {"I": 2.0, "Z": 3.0, "L": 5.0}
    assert lossy_list(s) == [("I", 2.0), ("Z", 3.0), ("L", 5.0)]


def test_rotations_with_loss():  # tests/loss.rs:279-331
    assert lossy_dict(run([("L", 1.0)], 1, [G.r1(G.RX, 0, 0.3)])) == {"L": 1.0}
    for word, partner in (("LZ", 1), ("ZL", 0)):
        a = run([(word, 1.0)], 2, [G.r2(G.RXX, 0, 1, 0.3)])
        b = run([(word, 1.0)], 2, [G.r1(G.RX, partner, 0.3)])
        assert lossy_dict(a) == lossy_dict(b)
    assert lossy_dict(run([("LL", 1.0)], 2, [G.r2(G.RXX, 0, 1, 0.3)])) == {"LL": 1.0}


def test_correlated_loss_channel():  # tests/loss.rs:333-385
    p = [0.1, 0.05, 0.2]
    ch = [G.correlated_loss_channel(0, 1, p)]
    assert lossy_dict(run([("ZI", 1.0)], 2, ch)) == {"ZI": 1.0 * (1.0 - 2.0 * p[1] - p[0])}
    assert lossy_dict(run([("ZL", 1.0)], 2, ch)) == {"ZL": 1.0 * (1.0 - p[2]), "ZI": p[1]}
    assert lossy_dict(run([("LZ", 1.0)], 2, ch)) == {"LZ": 1.0 * (1.0 - p[2]), "IZ": p[1]}
    assert lossy_dict(run([("LL", 1.0)], 2, ch)) == {"LL": 1.0, "IL": p[2], "LI": p[2], "II": p[0]}


def test_correlated_loss_ghz():  # tests/loss.rs:387-414
    p = [0.1, 0.0, 0.0]
    ops = [G.reset_loss_channel(0), G.reset_loss_channel(1), G.correlated_loss_channel(0, 1, p),
           G.g2(G.CNOT, 0, 1), G.g1(G.H, 0)]
    assert abs(run([("ZZ", 1.0)], 2, ops).trace("Z?*") - 1.0) < 1e-8
    assert abs(run([("XX", 1.0)], 2, ops).trace("Z?*") - 0.9) < 1e-8


def test_map_insert_multiple_order():
    # map_insert_multiple then consume (crates/ppvm-pauli-sum/src/sum/data.rs:180-189, 227-248):
    # the larger of (children, data) keeps its order and takes the other's entries.  One LL
    # term makes three children (more than the one data term): children order first
    s = run([("LL", 1.0)], 2, [G.correlated_loss_channel(0, 1, [0.1, 0.05, 0.2])])
    assert [w for w, _ in lossy_list(s)] == ["IL", "LI", "II", "LL"]
    # many data terms, one child: data order, the new key appended
    s = run([("ZI", 1.0), ("XX", 1.0), ("ZL", 1.0)], 2, [G.correlated_loss_channel(0, 1, [0.1, 0.05, 0.2])])
    assert [w for w, _ in lossy_list(s)] == ["ZI", "XX", "ZL"]
    assert lossy_dict(s)["ZI"] == 1.0 * (1.0 - 0.05 * 2.0 - 0.1) + 1.0 * 0.05


def test_lossy_sum_without_losses_matches_the_plain_sum():
    # the same circuit on a lossy sum with no lost qubit and on a plain sum: same terms, bits
    rng = np.random.default_rng(9)
    n = 70
    words = sorted({"".join(rng.choice(list("IXYZ"), n)) for _ in range(40)})
    terms = [(w, float(rng.uniform(-1, 1))) for w in words]
    ops = []
    for k in range(12):
        a, b = (int(v) for v in rng.choice(n, 2, replace=False))
        ops += [G.r1(G.RX, a, 0.3), G.g2(G.CNOT, a, b), G.r2(G.RZZ, a, b, 0.7), G.g1(G.H, b),
                G.depolarize2(a, b, 0.01), G.truncate()]
    a = lossy_oracle_from(terms, n, thr=1e-3)
    b = oracle_from(terms, n, thr=1e-3)
    a.run_ops(ops)
    b.run_ops(ops)
    ax, az, ac = a.export()
    bx, bz, bc = b.export()
    W = G.words(n)
    assert len(ac) == len(bc) > 100
    assert np.array_equal(ax[:, :W], bx) and np.array_equal(az[:, :W], bz)
    assert not ax[:, W:].any() and not az[:, W:].any()
    assert np.array_equal(ac.view(np.uint64), bc.view(np.uint64))


def test_generic_rotation_acts_on_the_qubits_that_are_not_lost():
    # pauli_rotation on a two-qubit generator reproduces rzz / rxx / ryy with their loss
    # fallback to a one-qubit rotation on the surviving qubit (crates/ppvm-pauli-sum/src/sum/rot2.rs:26-33)
    rng = np.random.default_rng(4)
    n = 5
    words = sorted({"".join(rng.choice(list("IXYZL"), n)) for _ in range(200)})
    terms = [(w, float(rng.uniform(-1, 1))) for w in words]
    for code, axis in ((G.RZZ, "Z"), (G.RXX, "X"), (G.RYY, "Y")):
        for a, b in ((0, 1), (3, 1), (2, 4)):
            lit = run(terms, n, [G.r2(code, a, b, 0.41)])
            gen = lossy_oracle_from(terms, n)
            w = ["I"] * n
            w[a] = w[b] = axis
            gx, gz = G.parse_lossy_word("".join(w), n)
            gen.pauli_rotation(gx, gz, 0.41)
            assert lossy_list(gen) == lossy_list(lit), (code, a, b)


def test_lossy_noise_skips_lost_qubits():
    # noise.rs:25 (pauli_error), :111 (depolarize1), :122 (depolarize2), :98-102 (two-qubit
    # error with a lost qubit), :138 (amplitude damping treats L as I)
    terms = [("LX", 1.0), ("XL", 1.0), ("LL", 1.0), ("XY", 1.0), ("ZI", 1.0)]
    s = run(terms, 2, [G.depolarize2(0, 1, 0.3)])
    d = lossy_dict(s)
    assert d["LX"] == d["XL"] == d["LL"] == 1.0 and d["XY"] == d["ZI"] == 1.0 - 0.3 * (16.0 / 15.0)
    s = lossy_oracle_from(terms, 2)
    s.two_qubit_pauli_error([0, 1], np.full(15, 0.01), truncate=False)
    d = lossy_dict(s)
    assert d["LX"] == d["XL"] == d["LL"] == 1.0 and d["XY"] != 1.0
    s = run([("L", 1.0), ("Z", 1.0)], 1, [G.pauli_error(0, (0.1, 0.1, 0.1)), G.depolarize1(0, 0.1),
                                          G.amplitude_damping(0, 0.3)])
    d = lossy_dict(s)
    assert d["L"] == 1.0 and set(d) == {"L", "Z", "I"}


def test_lossy_layout_round_trip():
    n = 130
    words = ["L" * n, "X" * 64 + "L" + "Z" * 65, "I" * n]
    x, z = lossy_planes(words, n)
    assert x.shape == (3, 6)
    assert [G.lossy_word_str(x[i], z[i], n) for i in range(3)] == words
    s = lossy_oracle_from([(w, 1.0) for w in words], n)
    assert list(lossy_dict(s)) == words
