"""ctypes binding of the CPU oracle (oracle/oracle.cpp) — TEST INFRASTRUCTURE ONLY.

Imported only by tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg,
always as the checker or the timed CPU reference, never by the product package.
"""

from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")


class OpStruct(ctypes.Structure):
    # Mirrors `ppvm_op` in include/ppvm_cuda.h.
    _fields_ = [
        ("code", ctypes.c_uint32),
        ("q0", ctypes.c_uint32),
        ("q1", ctypes.c_uint32),
        ("flags", ctypes.c_uint32),
        ("theta", ctypes.c_double),
        ("p", ctypes.c_double * 3),
    ]


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile if the library is missing."""
    if force or not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-C", _HERE], check=True, capture_output=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(LIB_PATH)
        vp, u32, u64, dbl, sz = (ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64,
                                 ctypes.c_double, ctypes.c_size_t)
        P64 = ctypes.POINTER(ctypes.c_uint64)
        PD = ctypes.POINTER(ctypes.c_double)
        L.oracle_create.restype = vp
        L.oracle_create.argtypes = [u32, dbl, u64, u32]
        L.oracle_create_sharded.restype = vp
        L.oracle_create_sharded.argtypes = [u32, dbl, u64, u32, ctypes.c_int]
        L.oracle_destroy.argtypes = [vp]
        L.oracle_clone.restype = vp
        L.oracle_clone.argtypes = [vp]
        L.oracle_words.restype = ctypes.c_int
        L.oracle_words.argtypes = [vp]
        L.oracle_set_max_loss_weight.argtypes = [vp, u64]
        L.oracle_len.restype = sz
        L.oracle_len.argtypes = [vp]
        L.oracle_add_terms.argtypes = [vp, P64, P64, PD, sz]
        L.oracle_set_preserve.argtypes = [vp, P64, P64, sz]
        L.oracle_run_ops.restype = ctypes.c_int
        L.oracle_run_ops.argtypes = [vp, ctypes.POINTER(OpStruct), sz, P64]
        L.oracle_pauli_rotation.argtypes = [vp, P64, P64, dbl]
        L.oracle_two_qubit_pauli_error.restype = ctypes.c_int
        L.oracle_two_qubit_pauli_error.argtypes = [vp, ctypes.POINTER(u32), sz, PD, ctypes.c_int]
        L.oracle_overlap_with_zero.restype = dbl
        L.oracle_overlap_with_zero.argtypes = [vp]
        L.oracle_trace.restype = ctypes.c_int
        L.oracle_trace.argtypes = [vp, ctypes.c_char_p, PD]
        L.oracle_overlap.restype = dbl
        L.oracle_overlap.argtypes = [vp, vp]
        L.oracle_export.restype = sz
        L.oracle_export.argtypes = [vp, P64, P64, PD, sz]
        _lib = L
    return _lib


def _p64(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))


def _pd(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def ops_to_struct(ops) -> ctypes.Array:
    """ops: sequence of (code, q0, q1, theta, (p0, p1, p2)) tuples."""
    arr = (OpStruct * max(1, len(ops)))()
    for i, (code, q0, q1, theta, p) in enumerate(ops):
        arr[i].code = code
        arr[i].q0 = q0
        arr[i].q1 = q1
        arr[i].flags = 0
        arr[i].theta = theta
        arr[i].p[0], arr[i].p[1], arr[i].p[2] = p
    return arr


class OracleSum:
    """The reference PauliSum semantics on the CPU.

    By default the IndexMap configuration (insertion-ordered map, one thread), the one every
    parity test compares against.  ``threads`` selects the reference's DashMap configuration
    instead, on that many host threads (0: all): the same terms and coefficients, in
    per-shard order.  ``lossy`` holds LossyPauliWord terms; their words cross this interface
    in the engine's lossy layout (2 * ceil(n/64) words per plane, loss bits in the X plane's
    upper half), and ``max_loss_weight`` is the strategy's MaxLossWeight."""

    def __init__(self, n_qubits: int, min_abs_coeff: float = 1e-10,
                 max_weight: int | None = None, clifford_angles: bool = False, threads: int | None = None,
                 lossy: bool = False, max_loss_weight: int | None = None):
        L = lib()
        self.n = n_qubits
        self.lossy = bool(lossy)
        mw = (1 << 64) - 1 if max_weight is None else int(max_weight)
        flags = (1 if clifford_angles else 0) | (4 if lossy else 0)
        if threads is None:
            self._h = L.oracle_create(n_qubits, min_abs_coeff, mw, flags)
        else:
            self._h = L.oracle_create_sharded(n_qubits, min_abs_coeff, mw, flags, int(threads))
        if not self._h:
            raise ValueError("oracle_create failed")
        self.W = L.oracle_words(self._h)
        if max_loss_weight is not None:
            L.oracle_set_max_loss_weight(self._h, int(max_loss_weight))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().oracle_destroy(h)
            self._h = None

    def clone(self) -> "OracleSum":
        o = OracleSum.__new__(OracleSum)
        o.n, o.W, o.lossy = self.n, self.W, self.lossy
        o._h = lib().oracle_clone(self._h)
        return o

    def __len__(self):
        return lib().oracle_len(self._h)

    def add_terms(self, x: np.ndarray, z: np.ndarray, c: np.ndarray):
        x = np.ascontiguousarray(x, dtype=np.uint64).reshape(-1, self.W)
        z = np.ascontiguousarray(z, dtype=np.uint64).reshape(-1, self.W)
        c = np.ascontiguousarray(c, dtype=np.float64).reshape(-1)
        lib().oracle_add_terms(self._h, _p64(x), _p64(z), _pd(c), len(c))

    def set_preserve(self, x: np.ndarray, z: np.ndarray):
        x = np.ascontiguousarray(x, dtype=np.uint64).reshape(-1, self.W)
        z = np.ascontiguousarray(z, dtype=np.uint64).reshape(-1, self.W)
        lib().oracle_set_preserve(self._h, _p64(x), _p64(z), x.shape[0])

    def run_ops(self, ops, counts: bool = False):
        arr = ops_to_struct(ops)
        cnt = np.zeros(max(1, len(ops)), dtype=np.uint64)
        rc = lib().oracle_run_ops(self._h, arr, len(ops), _p64(cnt) if counts else None)
        if rc != 0:
            raise ValueError(f"oracle op {rc - 1} rejected")
        return cnt[: len(ops)] if counts else None

    def pauli_rotation(self, gx: np.ndarray, gz: np.ndarray, theta: float):
        gx = np.ascontiguousarray(gx, dtype=np.uint64)
        gz = np.ascontiguousarray(gz, dtype=np.uint64)
        lib().oracle_pauli_rotation(self._h, _p64(gx), _p64(gz), theta)

    def two_qubit_pauli_error(self, pairs_flat, p, truncate: bool = True):
        """two_qubit_pauli_error_many over the flat pair list (noise.rs:39-105)."""
        t = np.ascontiguousarray(pairs_flat, dtype=np.uint32)
        pp = np.ascontiguousarray(p, dtype=np.float64)
        if pp.shape != (15,):
            raise ValueError("p needs 15 probabilities")
        rc = lib().oracle_two_qubit_pauli_error(self._h, t.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)),
                                                len(t), _pd(pp), 1 if truncate else 0)
        if rc != 0:
            raise ValueError("bad pair list")

    def overlap_with_zero(self) -> float:
        return lib().oracle_overlap_with_zero(self._h)

    def trace(self, pattern: str) -> float:
        out = ctypes.c_double(0.0)
        if lib().oracle_trace(self._h, pattern.encode(), ctypes.byref(out)) != 0:
            raise ValueError(f"bad pattern {pattern!r}")
        return out.value

    def overlap(self, other: "OracleSum") -> float:
        return lib().oracle_overlap(self._h, other._h)

    def export(self):
        n = len(self)
        x = np.zeros((max(n, 1), self.W), dtype=np.uint64)
        z = np.zeros((max(n, 1), self.W), dtype=np.uint64)
        c = np.zeros(max(n, 1), dtype=np.float64)
        lib().oracle_export(self._h, _p64(x), _p64(z), _pd(c), n)
        return x[:n], z[:n], c[:n]
