"""Learned truncation: a term-priority network and term-budget truncation on the GPU.

``TermPriorityNet`` wraps ``ppvm_mlp_*`` (include/ppvm_cuda.h): an 8 -> 64 -> 64 -> 1 GELU MLP
whose forward pass, backward pass and Adam step are hand-written kernels (BF16 tensor cores,
FP32 accumulation).  It predicts log10 |contribution of a term to <O>| from the term's
features (``PauliSum.features``), and ``PauliSum.truncate_budget(budget, net, ...)`` keeps
the ``budget`` terms it ranks highest.  Plain truncation at the same budget ranks by |c|.

Training labels come from the engine itself (``make_training_set``): terms sampled at every
layer of small lattice circuits are propagated, each on its own, through the layers that
remain (one batched run, ``PauliSumBatch``), and the label of a term is
log10(|c| * |<O> of the propagated term|).

No counterpart in the reference (it truncates by |coefficient| and weight only,
crates/ppvm-pauli-sum/src/strategy.rs:12-170).
"""

from __future__ import annotations

import ctypes
import math

import numpy as np

from . import circuits as C
from . import gates as G
from ._lib import EINVAL, OK, PPVMError, lib

N_PARAMS = 4801
LABEL_FLOOR = -12.0  # log10 of contributions at or below 1e-12


def _fp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


class TermPriorityNet:
    def __init__(self, seed: int = 0, device: int = 0):
        h = ctypes.c_void_p()
        self._h = None
        self._check(lib().ppvm_mlp_create(ctypes.byref(h), int(seed), int(device)))
        self._h = h

    def _check(self, st):
        if st != OK:
            msg = lib().ppvm_last_error_string().decode(errors="replace")
            raise ValueError(msg) if st == EINVAL else PPVMError(st, msg)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().ppvm_mlp_destroy(h)
            self._h = None

    @property
    def params(self) -> np.ndarray:
        p = np.zeros(N_PARAMS, dtype=np.float32)
        self._check(lib().ppvm_mlp_get_params(self._h, _fp(p), N_PARAMS))
        return p

    @params.setter
    def params(self, p) -> None:
        p = np.ascontiguousarray(p, dtype=np.float32)
        self._check(lib().ppvm_mlp_set_params(self._h, _fp(p), p.size))

    def train(self, feats, targets, epochs: int = 10, batch: int = 4096, lr: float = 2e-3, seed: int = 0) -> float:
        f = np.ascontiguousarray(feats, dtype=np.float32)
        t = np.ascontiguousarray(targets, dtype=np.float32)
        loss = ctypes.c_float()
        self._check(lib().ppvm_mlp_train(self._h, _fp(f), _fp(t), len(t), int(epochs), int(batch), float(lr),
                                         int(seed), ctypes.byref(loss)))
        return float(loss.value)

    def grad(self, feats, targets):
        f = np.ascontiguousarray(feats, dtype=np.float32)
        t = np.ascontiguousarray(targets, dtype=np.float32)
        g = np.zeros(N_PARAMS, dtype=np.float32)
        loss = ctypes.c_float()
        self._check(lib().ppvm_mlp_grad(self._h, _fp(f), _fp(t), len(t), _fp(g), ctypes.byref(loss)))
        return g, float(loss.value)

    def predict(self, feats) -> np.ndarray:
        f = np.ascontiguousarray(feats, dtype=np.float32)
        out = np.zeros(len(f), dtype=np.float32)
        self._check(lib().ppvm_mlp_predict(self._h, _fp(f), len(f), _fp(out)))
        return out


def split_layers(ops):
    """A Heisenberg gate list cut after every second TRUNCATE (one Trotter layer each)."""
    layers, cur, nt = [], [], 0
    for op in ops:
        cur.append(op)
        if op[0] == G.TRUNCATE:
            nt += 1
            if nt % 2 == 0:
                layers.append(cur)
                cur = []
    if cur:
        layers.append(cur)
    return layers


def make_training_set(L: int = 6, layers: int = 4, seeds=(11, 12, 13, 14), per_layer: int = 2048,
                      thr: float = 1e-7, label_thr: float = 1e-6, rng_seed: int = 0, device: int = 0):
    """(features [m, 8], labels [m]) from L x L kicked-Ising circuits with random angles.

    For each circuit the plain engine propagates the observable layer by layer at ``thr``;
    after layer l up to ``per_layer`` terms are drawn (uniformly) and each is propagated on
    its own through the remaining layers (a PauliSumBatch at ``label_thr``).  The label is
    log10(|c| |<O>_term|), floored at 1e-12."""
    from .batch import Instance, PauliSumBatch
    from .paulisum import PauliSum

    rng = np.random.default_rng(rng_seed)
    feats, labels = [], []
    for seed in seeds:
        wl = C.kicked_ising_random_h(L=L, layers=layers, seed=seed, thr=thr, obs=(L // 2, L // 2))
        lay = split_layers(wl.ops)
        s = PauliSum([wl.observable[0][0]], wl.n_qubits, [1.0], min_abs_coeff=thr, clifford_angles=True,
                     device=device)
        for li in range(len(lay) - 1):
            s.run(lay[li])
            left = len(lay) - 1 - li
            terms = s.terms
            f = s.features(L, left)
            pick = rng.choice(len(terms), size=min(per_layer, len(terms)), replace=False)
            rest = [op for part in lay[li + 1:] for op in part]
            insts = [Instance(wl.n_qubits, [(terms[int(i)][0], 1.0)], rest, label_thr, None) for i in pick]
            b = PauliSumBatch(insts, clifford_angles=True, device=device)
            b.run()
            o = b.overlap_with_zero()
            c = np.array([abs(terms[int(i)][1]) for i in pick])
            contrib = c * np.abs(o)
            labels.append(np.maximum(np.log10(np.maximum(contrib, 1e-300)), LABEL_FLOOR))
            feats.append(f[pick])
    return np.concatenate(feats).astype(np.float32), np.concatenate(labels).astype(np.float32)


def run_with_budget(wl, budget: int | None, net=None, lattice: int = 0, device: int = 0, digit_bits: int = 8):
    """Propagates ``wl`` layer by layer; between layers keeps ``budget`` terms (|c|, or the
    network's priority when ``net`` is given).  Returns (<O>, peak live terms)."""
    from .paulisum import PauliSum, ops_array

    lay = split_layers(wl.ops)
    s = PauliSum([wl.observable[0][0]], wl.n_qubits, [1.0], min_abs_coeff=wl.min_abs_coeff,
                 max_pauli_weight=wl.max_weight, clifford_angles=wl.clifford_angles, device=device)
    peak = 1
    for li, part in enumerate(lay):
        s.run(ops_array(part))
        peak = max(peak, len(s))
        left = len(lay) - 1 - li
        if budget is not None and left > 0:
            s.truncate_budget(budget, net, lattice, left, digit_bits)
    return s.overlap_with_zero(), peak


def compare_budgets(L: int = 10, layers: int = 4, seed: int = 2,
                    budgets=(500, 700, 1000, 1400, 2000, 2800, 4000, 5600, 8000, 1_000_000, 4_000_000),
                    train_L: int = 6, train_layers: int = 4, train_seeds=(11, 12, 13, 14, 15, 16, 17, 18),
                    per_layer: int = 2048, epochs: int = 300, label_thr: float = 1e-5, device: int = 0,
                    tol: float = 1e-3, log=None):
    """Learned vs plain term-budget truncation on the L x L kicked-Ising circuit with seeded
    angles U[0.4, 0.8], against the plain |c| < 1e-7 propagation without a budget."""
    import time

    def say(*a):
        if log:
            log(*a)

    t0 = time.perf_counter()
    X, y = make_training_set(L=train_L, layers=train_layers, seeds=train_seeds, per_layer=per_layer,
                             label_thr=label_thr, device=device)
    t_data = time.perf_counter() - t0
    say(f"training set: {len(y)} pairs in {t_data:.1f} s")
    net = TermPriorityNet(seed=7, device=device)
    t0 = time.perf_counter()
    loss = net.train(X, y, epochs=epochs, batch=512, lr=2e-3, seed=3)
    t_train = time.perf_counter() - t0
    say(f"trained: loss {loss:.4f} (label variance {float(np.var(y)):.4f}) in {t_train:.1f} s")
    wl = C.kicked_ising_random_h(L=L, layers=layers, seed=seed, thr=1e-7, obs=(L // 2, L // 2))
    run_with_budget(wl, None, device=device)  # warm-up
    t0 = time.perf_counter()
    ref, ref_peak = run_with_budget(wl, None, device=device)
    t_ref = time.perf_counter() - t0
    say(f"reference (|c| < 1e-7, no budget): <O> = {ref:.10f}, peak {ref_peak} terms, {t_ref:.3f} s")
    rows = []
    for B in budgets:
        for kind, nn in (("plain", None), ("learned", net)):
            run_with_budget(wl, B, nn, L, device=device)  # warm-up
            t0 = time.perf_counter()
            v, peak = run_with_budget(wl, B, nn, L, device=device)
            dt = time.perf_counter() - t0
            rows.append({"budget": int(B), "kind": kind, "O": v, "err": abs(v - ref), "s": dt, "peak": peak})
            say(f"budget {B:>9} {kind:>7}: <O> = {v:.10f} |err| = {abs(v - ref):.3e} {dt:.3f} s")

    def first_ok(kind):
        ok = [r for r in rows if r["kind"] == kind and r["err"] <= tol]
        return min(ok, key=lambda r: r["s"]) if ok else None

    return {"reference": {"O": ref, "s": t_ref, "peak": ref_peak}, "rows": rows,
            "train": {"pairs": int(len(y)), "data_s": t_data, "train_s": t_train, "loss": loss,
                      "label_var": float(np.var(y))},
            "time_to_tol": {"plain": first_ok("plain"), "learned": first_ok("learned"), "tol": tol}, "net": net}


__all__ = ["TermPriorityNet", "make_training_set", "run_with_budget", "split_layers", "N_PARAMS"]
