"""Pins the CPU oracle (oracle/oracle.cpp) to the reference's own golden values.

Every case cites the reference test it restates.  These run without a GPU.
"""

import json
import math
import os

import numpy as np
import pytest

from ppvm_b200 import gates as G
from tests.helpers import oracle_dict, oracle_from, oracle_list, planes

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_tables.json")))
UMAX = None  # no weight cap


def _signed(s):
    return (-1.0 if s[0] == "-" else 1.0), s.lstrip("+-")


OPS = {"x": G.X, "y": G.Y, "z": G.Z, "h": G.H, "s": G.S, "s_dag": G.S_DAG,
       "sqrt_x": G.SQRT_X, "sqrt_x_dag": G.SQRT_X_DAG, "sqrt_y": G.SQRT_Y,
       "sqrt_y_dag": G.SQRT_Y_DAG, "cnot": G.CNOT, "cz": G.CZ, "cy": G.CY}


@pytest.mark.parametrize("name", sorted(GOLD["phase_tables"]))
def test_clifford_sign_tables(name):
    # crates/ppvm-pauli-word/src/phase/clifford.rs:184-374 (signed tables)
    for inp, out in GOLD["phase_tables"][name]:
        si, wi = _signed(inp)
        so, wo = _signed(out)
        n = len(wi)
        s = oracle_from([(wi, si)], n, thr=0.0)
        code = OPS[name]
        s.run_ops([G.g1(code, 0)] if n == 1 else [G.g2(code, 0, 1)])
        assert oracle_dict(s) == {wo: so * si}, (name, inp, out)


@pytest.mark.parametrize("name", sorted(GOLD["word_tables"]))
def test_clifford_word_tables(name):
    # crates/ppvm-pauli-word/src/word/clifford.rs:7-179 (unsigned word maps)
    for inp, out in GOLD["word_tables"][name]:
        n = len(inp)
        s = oracle_from([(inp, 1.0)], n, thr=0.0)
        code = OPS[name]
        s.run_ops([G.g1(code, 0)] if n == 1 else [G.g2(code, 0, 1)])
        assert list(oracle_dict(s)) == [out]


def test_rot1_exact_children():
    # crates/ppvm-pauli-sum/src/sum/rot1.rs:186-251,279-310 at theta = 2.1
    t = 2.1
    c, s = math.cos(t), math.sin(t)
    cases = {
        G.RX: {"X": {"X": 1.0}, "Y": {"Y": c, "Z": -s}, "Z": {"Z": c, "Y": s}, "I": {"I": 1.0}},
        G.RY: {"X": {"X": c, "Z": s}, "Y": {"Y": 1.0}, "Z": {"Z": c, "X": -s}, "I": {"I": 1.0}},
        G.RZ: {"X": {"X": c, "Y": -s}, "Y": {"Y": c, "X": s}, "Z": {"Z": 1.0}, "I": {"I": 1.0}},
    }
    for code, table in cases.items():
        for w, want in table.items():
            o = oracle_from([(w, 1.0)], 1, thr=0.0)
            o.run_ops([G.r1(code, 0, t)])
            assert oracle_dict(o) == want, (G.NAMES[code], w)


def test_r_axis_angle_is_heisenberg_ordered():
    # rot1.rs:253-277: r(0, th) == rx(th); r(pi/2, th) == ry(th) (not ry(-th))
    t = 2.1
    for phi, code in ((0.0, G.RX), (math.pi / 2, G.RY)):
        a = oracle_from([("Z", 1.0)], 1, thr=0.0)
        a.run_ops([G.r1(G.RZ, 0, phi), G.r1(G.RX, 0, t), G.r1(G.RZ, 0, -phi)])
        b = oracle_from([("Z", 1.0)], 1, thr=0.0)
        b.run_ops([G.r1(code, 0, t)])
        assert abs(a.overlap(b) - 1.0) < 1e-9


@pytest.mark.parametrize("code,axis", [(G.RXX, (1, 0)), (G.RYY, (1, 1)), (G.RZZ, (0, 1))])
def test_rot2_fast_paths_match_generic(code, axis):
    # crates/ppvm-pauli-sum/src/sum/rot2.rs:266-299: fast path == generic rotate_2 at 0.7,
    # and rot2.rs:331-350 non-adjacent addressing (qubits 0 and 2).
    t = 0.7
    for n, (a, b) in ((2, (0, 1)), (3, (0, 2))):
        for p in "IXYZ":
            for q in "IXYZ":
                w = p + ("I" if n == 3 else "") + q
                fast = oracle_from([(w, 1.0)], n, thr=0.0)
                fast.run_ops([G.r2(code, a, b, t)])
                gen = oracle_from([(w, 1.0)], n, thr=0.0)
                gx = np.zeros(1, dtype=np.uint64)
                gz = np.zeros(1, dtype=np.uint64)
                for qq in (a, b):
                    if axis[0]:
                        gx[0] |= np.uint64(1 << qq)
                    if axis[1]:
                        gz[0] |= np.uint64(1 << qq)
                gen.pauli_rotation(gx, gz, t)
                assert oracle_dict(fast) == oracle_dict(gen), (G.NAMES[code], w)


def test_rzz_explicit_values():
    # rot2.rs:303-327
    t = 0.7
    s = oracle_from([("XI", 1.0)], 2, thr=0.0)
    s.run_ops([G.r2(G.RZZ, 0, 1, t)])
    assert oracle_dict(s) == {"XI": math.cos(t), "YZ": -math.sin(t)}
    s = oracle_from([("YI", 1.0)], 2, thr=0.0)
    s.run_ops([G.r2(G.RZZ, 0, 1, t)])
    assert oracle_dict(s) == {"YI": math.cos(t), "XZ": math.sin(t)}
    s = oracle_from([("ZZ", 1.0)], 2, thr=0.0)
    s.run_ops([G.r2(G.RZZ, 0, 1, t)])
    assert oracle_dict(s) == {"ZZ": 1.0}


def _trotter_ops(n=4, steps=10, theta_x=0.1, theta_zz=0.0125, noise=(2.5e-5,) * 3):
    # crates/ppvm-pauli-sum/tests/trotter.rs:35-54 (truncate after every op)
    ops = []
    for _ in range(steps):
        for i in range(n):
            ops += [G.pauli_error(i, noise), G.truncate(), G.r1(G.RX, i, theta_x), G.truncate()]
        for i in range(n - 1):
            ops += [G.pauli_error(i + 1, noise), G.truncate(), G.pauli_error(i, noise),
                    G.truncate(), G.r2(G.RZZ, i, i + 1, theta_zz), G.truncate()]
    return ops


def _expect_on_zero(s):
    # trotter.rs:58-68: sum of coefficients of words made of I and Z only
    return sum(c for w, c in oracle_list(s) if set(w) <= {"I", "Z"})


def test_trotter_golden():
    # crates/ppvm-pauli-sum/tests/trotter.rs:80-121
    n = 4
    seed = [("".join("Z" if i == j else "I" for i in range(n)), 1.0) for j in range(n)]
    exact = oracle_from(seed, n, thr=0.0)
    exact.run_ops(_trotter_ops())
    ev = _expect_on_zero(exact)
    assert abs(ev - GOLD["golden_trotter_n4"]) < 1e-9
    assert abs(exact.overlap_with_zero() - ev) < 1e-12
    approx = oracle_from(seed, n, thr=1e-6)
    approx.run_ops(_trotter_ops())
    assert abs(ev - _expect_on_zero(approx)) < 1e-6


def test_cnot_golden():
    # crates/ppvm-pauli-sum/tests/cnot.rs:7-28
    s = oracle_from([("ZZ", 1.0)], 2, thr=0.0)
    s.run_ops([G.r1(G.RZ, 0, 1.1), G.r1(G.RY, 0, 2.1), G.r1(G.RZ, 0, 1.1),
               G.r1(G.RZ, 1, 1.1), G.r1(G.RY, 1, 2.1), G.r1(G.RZ, 1, 1.1),
               G.g2(G.CNOT, 0, 1), G.r1(G.RX, 0, 2.1), G.r1(G.RX, 1, 2.1)])
    v = s.trace("Z?*")
    assert math.isclose(v, GOLD["golden_cnot"], rel_tol=1e-12)


def test_ghz():
    # crates/ppvm-pauli-sum/tests/ghz.rs
    s = oracle_from([("Y", 1.0)], 1, thr=0.0)
    s.run_ops([G.g1(G.H, 0)])
    assert oracle_list(s) == [("Y", -1.0)]
    s = oracle_from([("ZI", 1.0), ("IZ", 1.0), ("ZZ", 1.0), ("II", 1.0)], 2, thr=0.0)
    s.run_ops([G.g1(G.H, 0), G.g2(G.CNOT, 0, 1)])
    assert oracle_dict(s) == {"XX": 1.0, "YY": -1.0, "ZZ": 1.0, "II": 1.0}
    s = oracle_from([("ZZ", 1.0)], 2, thr=0.0)
    s.run_ops([G.g2(G.CNOT, 0, 1), G.g1(G.H, 0)])
    assert s.trace("Z?*") == 1.0


def test_strategies():
    # crates/ppvm-pauli-sum/tests/strategy.rs:9-91
    s = oracle_from([("ZZ", 1.0), ("XX", 1e-3), ("YY", 1e-5), ("XZ", -0.5)], 2, thr=1e-4)
    s.run_ops([G.truncate()])
    assert oracle_list(s) == [("ZZ", 1.0), ("XX", 1e-3), ("XZ", -0.5)]
    s = oracle_from([("XXX", 1.0), ("ZZI", 1e-4), ("YZY", -10.0), ("IXX", -0.1)], 3, thr=0.0, maxw=2)
    s.run_ops([G.truncate()])
    assert oracle_list(s) == [("ZZI", 1e-4), ("IXX", -0.1)]
    terms = [("ZZI", 1.0), ("XIX", 1e-3), ("IYY", 1e-5), ("XIZ", -0.5), ("XXX", 1.0),
             ("ZIZ", 1e-4), ("YZY", -10.0), ("IXX", -0.1)]
    s = oracle_from(terms, 3, thr=1e-4, maxw=2)
    s.run_ops([G.truncate()])
    assert oracle_dict(s) == {"ZZI": 1.0, "XIX": 1e-3, "XIZ": -0.5, "ZIZ": 1e-4, "IXX": -0.1}
    # |c| == thr is kept, exact 0.0 dropped for thr > 0 (strict `abs < thr`, coefficient.rs:59-62)
    s = oracle_from([("X", 1e-4), ("Z", 0.0)], 1, thr=1e-4)
    s.run_ops([G.truncate()])
    assert oracle_list(s) == [("X", 1e-4)]


def test_deferred_truncation_semantics():
    # crates/ppvm-pauli-sum/tests/truncation_semantics.rs:34-79
    tau, th = 0.05, 0.03
    a = oracle_from([("Z", 1.0)], 1, thr=tau)
    a.run_ops([G.r1(G.RX, 0, th), G.r1(G.RX, 0, th), G.truncate()])
    e = oracle_from([("Z", 1.0)], 1, thr=0.0)
    e.run_ops([G.r1(G.RX, 0, th), G.r1(G.RX, 0, th)])
    ref = {w: c for w, c in oracle_dict(e).items() if abs(c) >= tau}
    assert "Y" in ref
    assert oracle_dict(a) == ref


def test_preserve_strings():
    # crates/ppvm-pauli-sum/tests/preserve.rs:33-114
    n = 3
    single = ["".join("Z" if i == j else "I" for i in range(n)) for j in range(n)]
    s = oracle_from([("ZII", 1e-6), ("IZI", 1e-6), ("IIZ", 1e-6), ("XYZ", 1e-6), ("XXX", 0.7)], n, thr=0.5)
    s.set_preserve(*planes(single, n))
    s.run_ops([G.truncate()])
    kept = oracle_dict(s)
    assert set(kept) == {"ZII", "IZI", "IIZ", "XXX"}
    # re-inserted preserved strings go to the end, in iteration order (data.rs:300-310)
    assert [w for w, _ in oracle_list(s)] == ["XXX", "ZII", "IZI", "IIZ"]
    n = 4
    single = ["".join("Z" if i == j else "I" for i in range(n)) for j in range(n)]
    s = oracle_from([(w, 1.0) for w in single], n, thr=0.5)
    s.set_preserve(*planes(single, n))
    for a, b in ((0, 1), (1, 2), (2, 3)):
        s.run_ops([G.r2(G.RXX, a, b, 0.37), G.r2(G.RYY, a, b, 0.37), G.truncate()])
    d = oracle_dict(s)
    for w in single:
        assert abs(d[w] - 1.0) < 1e-10


def test_python_basics():
    # ppvm-python/test/test_basics.py:8-38 (truncate after every call, default 1e-10)
    s = oracle_from([("ZZ", 1.0)], 2)
    s.run_ops([G.g2(G.CNOT, 0, 1), G.truncate(), G.g1(G.H, 0), G.truncate()])
    assert oracle_list(s) == [("IZ", 1.0)]
    assert s.overlap_with_zero() == 1.0
    n, w = 200, 80
    terms = [("".join("Z" if i == j else "I" for i in range(n)), 1.0) for j in range(n)]
    s = oracle_from(terms, n, maxw=w)
    ops = []
    for i in reversed(range(1, n)):
        ops += [G.g2(G.CNOT, i - 1, i), G.truncate()]
    ops += [G.g1(G.H, 0), G.truncate()]
    s.run_ops(ops)
    assert s.overlap_with_zero() == 0.0


def test_trace_patterns():
    # crates/ppvm-pauli-word/src/pattern/contains.rs:153-214 ("Z?*" rejects XYY)
    s = oracle_from([("XYY", 2.0), ("ZIZ", 3.0), ("III", 5.0), ("IXI", 7.0)], 3, thr=0.0)
    assert s.trace("Z?*") == 8.0
    assert s.trace("X0Y1Y2") == 2.0
    assert s.trace("[XY]*") == 5.0 + 2.0
    assert s.trace("X1") == 7.0
