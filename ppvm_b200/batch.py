"""``PauliSumBatch``: many independent PauliSums advanced together on one GPU.

Each instance has its own qubit count, truncation strategy, initial terms and gate list (in
Heisenberg order, with TRUNCATE ops as ``ppvm_b200.gates`` builds them).  The whole batch
runs with one CTA per instance and one launch per Trotter layer (CUDA graphs), through
``ppvm_batch_*`` in include/ppvm_cuda.h.  Every instance's result is what a ``PauliSum``
with ``exact_order=True`` gives for the same list: same terms, same order, same
coefficients.  The reference has no batch object; its users loop over PauliSums
(crates/ppvm-pauli-sum/benches/trotter.rs:28-44).
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import gates as G
from ._lib import EINVAL, FLAG_CLIFFORD_ANGLES, OK, UMAX, Op, PPVMError, lib
from .paulisum import GateList, _p64, _pd, ops_array


@dataclass
class Instance:
    n_qubits: int
    terms: list  # [(word, coeff)]
    ops: list    # gate tuples, or a GateList packed once with ops_array
    min_abs_coeff: float = 1e-10
    max_pauli_weight: int | None = None


class PauliSumBatch:
    def __init__(self, instances: list[Instance], *, clifford_angles: bool = False, device: int = 0,
                 capacity=None):
        if not instances:
            raise ValueError("a batch needs at least one instance")
        k = len(instances)
        nq = (ctypes.c_uint32 * k)(*[int(i.n_qubits) for i in instances])
        thr = (ctypes.c_double * k)(*[float(i.min_abs_coeff) for i in instances])
        mw = (ctypes.c_uint64 * k)(*[UMAX if i.max_pauli_weight is None else int(i.max_pauli_weight)
                                     for i in instances])
        h = ctypes.c_void_p()
        self._h = None
        self._check(lib().ppvm_batch_create(ctypes.byref(h), k, nq, thr, mw,
                                            FLAG_CLIFFORD_ANGLES if clifford_angles else 0, device))
        self._h = h
        self.instances = instances
        lists = []
        for j, inst in enumerate(instances):
            if inst.terms:
                W = G.words(inst.n_qubits)
                x = np.zeros((len(inst.terms), W), dtype=np.uint64)
                z = np.zeros((len(inst.terms), W), dtype=np.uint64)
                for t, (w, _) in enumerate(inst.terms):
                    x[t], z[t] = G.parse_word(w, inst.n_qubits)
                c = np.array([float(cf) for _, cf in inst.terms], dtype=np.float64)
                self._check(lib().ppvm_batch_add_terms(self._h, j, _p64(x), _p64(z), _pd(c), len(c)))
            lists.append(inst.ops if isinstance(inst.ops, GateList) else ops_array(inst.ops))
        # every list in one call: the library packs them on several host threads
        ptrs = (ctypes.POINTER(Op) * k)(*[gl.ptr for gl in lists])
        counts = (ctypes.c_size_t * k)(*[len(gl) for gl in lists])
        self._check(lib().ppvm_batch_set_ops_all(self._h, ptrs, counts))
        if capacity is not None:
            caps = np.ascontiguousarray(capacity, dtype=np.uint64)
            if caps.shape != (k,):
                raise ValueError("capacity needs one value per instance")
            self._check(lib().ppvm_batch_reserve(self._h, _p64(caps)))

    @classmethod
    def from_workloads(cls, workloads, **kw) -> "PauliSumBatch":
        return cls([Instance(w.n_qubits, list(w.observable), list(w.ops), w.min_abs_coeff, w.max_weight)
                    for w in workloads], **kw)

    def _check(self, st: int) -> None:
        if st != OK:
            msg = lib().ppvm_last_error_string().decode(errors="replace")
            raise ValueError(msg) if st == EINVAL else PPVMError(st, msg)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().ppvm_batch_destroy(h)
            self._h = None

    def __len__(self) -> int:
        return len(self.instances)

    def set_stream(self, stream_handle: int | None) -> None:
        self._check(lib().ppvm_batch_set_stream(self._h, ctypes.c_void_p(stream_handle or 0)))

    def run(self) -> None:
        """Every instance from its initial terms through its whole list (layer graphs)."""
        self._check(lib().ppvm_batch_run(self._h))

    def run_persistent(self) -> None:
        """The same in one launch (each CTA runs its instance's whole list)."""
        self._check(lib().ppvm_batch_run_persistent(self._h))

    def capacities(self) -> np.ndarray:
        """Term capacity of every instance (after a run: at least its peak live count)."""
        caps = np.zeros(len(self), dtype=np.uint64)
        self._check(lib().ppvm_batch_get_capacity(self._h, _p64(caps)))
        return caps

    def set_config(self, block: int, items: int, table_factor: int) -> None:
        self._check(lib().ppvm_batch_set_config(self._h, block, items, table_factor))

    def config(self) -> dict:
        b, i, t = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        self._check(lib().ppvm_batch_get_config(self._h, ctypes.byref(b), ctypes.byref(i), ctypes.byref(t)))
        return {"block": b.value, "items": i.value, "table_factor": t.value}

    def autotune(self) -> dict:
        """Times every launch configuration on this batch and keeps the fastest."""
        b, i, t, ms = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
        self._check(lib().ppvm_batch_autotune(self._h, ctypes.byref(b), ctypes.byref(i), ctypes.byref(t),
                                              ctypes.byref(ms)))
        return {"block": b.value, "items": i.value, "table_factor": t.value, "best_ms": ms.value}

    def overlap_with_zero(self) -> np.ndarray:
        out = np.zeros(len(self), dtype=np.float64)
        self._check(lib().ppvm_batch_overlap_with_zero(self._h, _pd(out)))
        return out

    def len_of(self, j: int) -> int:
        n = ctypes.c_size_t()
        self._check(lib().ppvm_batch_len(self._h, j, ctypes.byref(n)))
        return int(n.value)

    def export(self, j: int):
        n = self.len_of(j)
        W = G.words(self.instances[j].n_qubits)
        x = np.zeros((max(n, 1), W), dtype=np.uint64)
        z = np.zeros((max(n, 1), W), dtype=np.uint64)
        c = np.zeros(max(n, 1), dtype=np.float64)
        got = ctypes.c_size_t()
        self._check(lib().ppvm_batch_export_terms(self._h, j, _p64(x), _p64(z), _pd(c), n, ctypes.byref(got)))
        return x[:n], z[:n], c[:n]

    def terms(self, j: int) -> list[tuple[str, float]]:
        x, z, c = self.export(j)
        n = self.instances[j].n_qubits
        return [(G.word_str(x[i], z[i], n), float(c[i])) for i in range(len(c))]

    def transfer_counters(self) -> tuple[int, int]:
        """Bytes copied host->device and device->host by this batch since it was created."""
        h2d, d2h = ctypes.c_uint64(), ctypes.c_uint64()
        self._check(lib().ppvm_batch_transfer_counters(self._h, ctypes.byref(h2d), ctypes.byref(d2h)))
        return int(h2d.value), int(d2h.value)

    def term_gate_updates(self):
        per = np.zeros(len(self), dtype=np.uint64)
        tot = ctypes.c_uint64()
        self._check(lib().ppvm_batch_term_gate_updates(self._h, _p64(per), ctypes.byref(tot)))
        return per, int(tot.value)


__all__ = ["Instance", "PauliSumBatch"]
