"""Synthetic workloads of the PauliSum path, as Heisenberg-ordered gate lists.

Each generator returns a ``Workload``: qubit count, truncation strategy, the observable,
and the op list in Heisenberg order (the exact reverse of the forward circuit) with
explicit ``TRUNCATE`` ops where a Python caller of the reference would truncate (once per
gate-list call, crates/ppvm-python-native/src/interface.rs:156-310).  The same list drives
the GPU engine, the CPU oracle and the benchmark, so all share the term-gate-updates count.

Random choices use splitmix64 seeded per workload, so lists are reproducible everywhere.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

from . import gates as G

MASK64 = (1 << 64) - 1


class SplitMix64:
    def __init__(self, seed: int):
        self.s = seed & MASK64

    def next(self) -> int:
        self.s = (self.s + 0x9E3779B97F4A7C15) & MASK64
        z = self.s
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK64
        return z ^ (z >> 31)

    def uniform(self) -> float:
        return (self.next() >> 11) * (1.0 / (1 << 53))

    def below(self, k: int) -> int:
        return self.next() % k

    def uniform_range(self, a: float, b: float) -> float:
        return a + (b - a) * self.uniform()

    def int_range(self, lo: int, hi: int) -> int:  # inclusive
        return lo + self.below(hi - lo + 1)


@dataclass
class Workload:
    name: str
    n_qubits: int
    min_abs_coeff: float
    max_weight: int | None
    observable: list[tuple[str, float]]
    ops: list = field(default_factory=list)
    clifford_angles: bool = False
    meta: dict = field(default_factory=dict)

    @property
    def n_gates(self) -> int:
        return sum(1 for op in self.ops if op[0] != G.TRUNCATE)


def _z_word(n: int, q: int) -> str:
    return "".join("Z" if i == q else "I" for i in range(n))


def tfim_1d(n: int = 20, J: float = 1.0, h: float = 1.0, dt: float = 0.1, steps: int = 10,
            thr: float = 1e-4, obs_qubit: int | None = None) -> Workload:
    """Open-chain transverse-field Ising Trotter circuit.  Forward step: RZZ(i, i+1; 2 J dt)
    on every bond, then RX(i; 2 h dt) on every qubit; Heisenberg order reverses the whole list;
    TRUNCATE after each layer half."""
    tzz, tx = 2 * J * dt, 2 * h * dt
    q_obs = n // 2 if obs_qubit is None else obs_qubit
    ops = []
    for _ in range(steps):
        ops += [G.r1(G.RX, i, tx) for i in reversed(range(n))] + [G.truncate()]
        ops += [G.r2(G.RZZ, i, i + 1, tzz) for i in reversed(range(n - 1))] + [G.truncate()]
    return Workload(f"tfim1d_n{n}_steps{steps}", n, thr, None, [(_z_word(n, q_obs), 1.0)], ops,
                    meta={"J": J, "h": h, "dt": dt, "steps": steps})


def lattice_bonds(L: int) -> list[tuple[int, int]]:
    """Open LxL square lattice, qubit (r, c) = r*L + c; horizontal bonds then vertical, row-major."""
    hb = [(r * L + c, r * L + c + 1) for r in range(L) for c in range(L - 1)]
    vb = [(r * L + c, (r + 1) * L + c) for r in range(L - 1) for c in range(L)]
    return hb + vb


def kicked_ising_2d(L: int = 12, layers: int = 20, theta_h=0.6, theta_zz: float = -math.pi / 2,
                    thr: float = 1e-5, max_weight: int | None = 10, obs=None) -> Workload:
    """2D kicked Ising: each forward layer applies RX(theta_h) on every qubit, then RZZ(theta_zz)
    on all bonds.  theta_h may be a per-layer list.  At theta_zz = -pi/2 the RZZ layer is
    Clifford (``clifford_angles``).  Observable: Z at site ``obs`` (default the centre,
    (L//2, L//2), which is (6, 6) on the 12 x 12 lattice)."""
    n = L * L
    obs = (L // 2, L // 2) if obs is None else tuple(obs)
    if not (0 <= obs[0] < L and 0 <= obs[1] < L):
        raise ValueError(f"observable site {obs} is outside the {L}x{L} lattice")
    bonds = lattice_bonds(L)
    th = list(theta_h) if isinstance(theta_h, (list, tuple)) else [theta_h] * layers
    ops = []
    for layer in reversed(range(layers)):
        ops += [G.r2(G.RZZ, a, b, theta_zz) for a, b in reversed(bonds)] + [G.truncate()]
        ops += [G.r1(G.RX, q, th[layer]) for q in reversed(range(n))] + [G.truncate()]
    q_obs = obs[0] * L + obs[1]
    return Workload(f"kicked_ising_{L}x{L}_layers{layers}", n, thr, max_weight, [(_z_word(n, q_obs), 1.0)],
                    ops, clifford_angles=abs(abs(theta_zz) - math.pi / 2) < 1e-15,
                    meta={"L": L, "layers": layers, "bonds": len(bonds)})


def kicked_ising_random_h(L: int = 10, layers: int = 30, seed: int = 2, lo: float = 0.4, hi: float = 0.8,
                          thr: float = 1e-7, max_weight: int | None = None, obs=None) -> Workload:
    """2D kicked Ising with a seeded transverse angle per layer, theta_h ~ U[lo, hi]
    (splitmix64), RZZ(-pi/2) on every bond; observable Z at ``obs``."""
    rng = SplitMix64(seed)
    th = [rng.uniform_range(lo, hi) for _ in range(layers)]
    wl = kicked_ising_2d(L=L, layers=layers, theta_h=th, thr=thr, max_weight=max_weight, obs=obs)
    wl.name = f"kicked_ising_{L}x{L}_layers{layers}_seed{seed}"
    wl.meta["theta_h"] = th
    return wl


def clifford_t(n: int = 64, layers: int = 1000, seed: int = 0, p_t: float = 0.05, thr: float = 1e-6,
               heisenberg_layers: int | None = None) -> Workload:
    """Random Clifford+T brickwork.  Forward layer: each qubit one of {H, S, S_DAG}; CNOT on
    (2i, 2i+1) for even layers, (2i+1, 2i+2) for odd ones; then T = RZ(pi/4) on each qubit with
    probability p_t.  Observable: a random weight-4 Pauli.  Heisenberg order, TRUNCATE after
    each layer's T block (Cliffords keep |c|, so a truncate after them is a no-op).

    ``heisenberg_layers`` = k keeps only the first k layers of the Heisenberg list (the last k
    forward layers): a prefix of the same ``layers``-layer circuit, observable included."""
    rng = SplitMix64(seed)
    fwd_layers = []
    for layer in range(layers):
        singles = [(G.H, G.S, G.S_DAG)[rng.below(3)] for _ in range(n)]
        start = 0 if layer % 2 == 0 else 1
        pairs = [(a, a + 1) for a in range(start, n - 1, 2)]
        ts = [q for q in range(n) if rng.uniform() < p_t]
        fwd_layers.append((singles, pairs, ts))
    qs = []
    while len(qs) < 4:
        q = rng.below(n)
        if q not in qs:
            qs.append(q)
    word = ["I"] * n
    for q in qs:
        word[q] = "XYZ"[rng.below(3)]
    kept = list(reversed(fwd_layers))
    if heisenberg_layers is not None:
        kept = kept[:heisenberg_layers]
    ops = []
    for singles, pairs, ts in kept:
        ops += [G.r1(G.RZ, q, math.pi / 4) for q in reversed(ts)] + [G.truncate()]
        ops += [G.g2(G.CNOT, a, b) for a, b in reversed(pairs)]
        ops += [G.g1(code, q) for q, code in reversed(list(enumerate(singles)))]
    name = f"clifford_t_n{n}_layers{layers}_seed{seed}"
    if heisenberg_layers is not None:
        name += f"_first{len(kept)}"
    return Workload(name, n, thr, None, [("".join(word), 1.0)], ops,
                    meta={"layers": layers, "seed": seed, "heisenberg_layers": len(kept),
                          "t_gates": sum(len(t) for _, _, t in kept)})


def batched_tfim(count: int = 256, seed: int = 1, thr: float = 1e-5) -> list[Workload]:
    """Independent 1D TFIM instances: n ~ U[16,128], steps ~ U[5,30], h ~ U[0.5,1.5], J = 1,
    dt = 0.05, observable Z on qubit n/2."""
    rng = SplitMix64(seed)
    out = []
    for _ in range(count):
        n = rng.int_range(16, 128)
        steps = rng.int_range(5, 30)
        h = rng.uniform_range(0.5, 1.5)
        out.append(tfim_1d(n=n, J=1.0, h=h, dt=0.05, steps=steps, thr=thr, obs_qubit=n // 2))
    return out


def term_gate_updates(live_counts, ops) -> int:
    """Sum over gates (TRUNCATE excluded) of the live terms entering the gate."""
    return int(sum(int(c) for c, op in zip(live_counts, ops) if op[0] != G.TRUNCATE))
