"""The benchmarked workloads in full against the oracle, through the C ABI.

The 12x12 kicked-Ising circuit of the headline bench line (20 layers, RX(0.6) then
RZZ(-pi/2) on 264 bonds per layer, obs Z(6,6), |c| < 1e-5, weight cap 10) is propagated by
the GPU engine in both term-order modes and by the oracle, layer by layer.  After every layer
the term sets must be identical with every coefficient equal bit for bit (and the term lists
identical in order with ``exact_order``), the live count entering every gate must equal the
oracle's, and <O> must agree to 1e-10.  The same holds for the deepest prefixes of the
Clifford+T circuit (n=64, 1000 layers, seed 0) that the oracle finishes in about a minute.
"""

import numpy as np
import pytest

from ppvm_b200 import circuits as C
from ppvm_b200 import gates as G
from tests.helpers import oracle_from
from tests.test_gpu_parity import gpu_from, same, same_set

pytestmark = pytest.mark.gpu


def layers_of(ops, truncates_per_layer=2):
    """Splits a Heisenberg gate list into layers: a cut after every ``truncates_per_layer``-th
    TRUNCATE (two for kicked Ising, one per layer half; one for Clifford+T)."""
    out, cur, seen = [], [], 0
    for op in ops:
        cur.append(op)
        if op[0] == G.TRUNCATE:
            seen += 1
            if seen % truncates_per_layer == 0:
                out.append(cur)
                cur = []
    if cur:
        out.append(cur)
    return out


def lockstep(wl, chunks, modes=(False, True)):
    gs = {exact: gpu_from(wl.observable, wl.n_qubits, wl.min_abs_coeff, wl.max_weight, wl.clifford_angles,
                          exact=exact) for exact in modes}
    o = oracle_from(wl.observable, wl.n_qubits, wl.min_abs_coeff, wl.max_weight, wl.clifford_angles)
    updates = 0
    for chunk in chunks:
        want = o.run_ops(chunk, counts=True)
        for exact, g in gs.items():
            g.run(chunk)
            assert np.array_equal(g.live_counts(), want)
            (same if exact else same_set)(g, o)
        updates += C.term_gate_updates(want, chunk)
    owz = o.overlap_with_zero()
    for g in gs.values():
        assert abs(g.overlap_with_zero() - owz) < 1e-10
    return updates, owz, len(o)


def test_kicked_ising_12x12_full_headline_workload():
    wl = C.kicked_ising_2d(L=12, layers=20, theta_h=0.6, thr=1e-5, max_weight=10)
    updates, owz, n = lockstep(wl, layers_of(wl.ops))
    # the figures the bench line reports for this workload
    assert updates == 943844417
    assert n > 0 and abs(owz - 3.9233401326421296e-05) < 1e-10


@pytest.mark.parametrize("exact", [False, True])
def test_clifford_t_first_24_layers(exact):
    wl = C.clifford_t(heisenberg_layers=24)
    updates, _, n = lockstep(wl, layers_of(wl.ops, 1), modes=(exact,))
    assert updates == 88755388 and n == 590976


def test_clifford_t_first_26_layers():
    # 5.1e6 live terms at the end (the config-3 bench workload): one comparison at the end
    wl = C.clifford_t(heisenberg_layers=26)
    chunks = layers_of(wl.ops, 1)
    updates, _, n = lockstep(wl, [sum(chunks[:-1], []), chunks[-1]], modes=(False,))
    assert updates == 806335036 and n == 5132160
