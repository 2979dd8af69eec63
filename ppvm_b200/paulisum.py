"""``PauliSum``: the reference's Python PauliSum API over the B200 engine.

Mirrors ``ppvm.PauliSum`` (ppvm-python/src/ppvm/paulisum.py:79-499 and the gate mixins of
ppvm-python/src/ppvm/mixins.py in the reference): same constructor fields, the ``new``
shorthand, gate names and aliases, target broadcasting (variadic indices or one sequence;
two-qubit gates take flat pairs), the ``truncate: bool = True`` kwarg on every gate, and the
readouts ``overlap_with_zero``, ``overlap``, ``trace``, ``terms``, ``weights``,
``current_max_weight``.  Gates must be applied in reverse circuit order (Heisenberg picture).

Every call goes through the C ABI of include/ppvm_cuda.h; the terms live on the GPU.
Argument errors raise ``ValueError`` like the reference binding
(crates/ppvm-python-native/src/lib.rs:12-22); device failures raise ``PPVMError``.
"""

from __future__ import annotations

import ctypes
import math
import re
from collections.abc import Iterable, Sequence
from typing import Any

import numpy as np

from . import gates as G
from ._lib import EINVAL, FLAG_CLIFFORD_ANGLES, FLAG_EXACT_ORDER, FLAG_LOSSY, OK, UMAX, Op, PPVMError, lib

_COMPACT_RE = re.compile(r"^([IXYZ]\d+)+$")
_COMPACT_TOKEN_RE = re.compile(r"([IXYZ])(\d+)")


def _parse_term(term, n_qubits: int):
    """``"IX"``, ``"X1"`` (compact: Pauli at index) or ``(str, coeff)``."""
    s, coeff = term if isinstance(term, tuple) else (term, 1.0)
    if _COMPACT_RE.match(s):
        chars = ["I"] * n_qubits
        for pauli, idx in _COMPACT_TOKEN_RE.findall(s):
            i = int(idx)
            if i >= n_qubits:
                raise ValueError(f"Qubit index {i} out of range for {n_qubits}-qubit system.")
            chars[i] = pauli
        s = "".join(chars)
    return s, float(coeff)


def _is_seq(obj) -> bool:
    if isinstance(obj, (list, tuple)):
        return True
    if isinstance(obj, (int, str, bytes)):
        return False
    return isinstance(obj, Iterable)


def _targets(args) -> list[int]:
    if len(args) == 1 and _is_seq(args[0]):
        args = args[0]
    return [int(a) for a in args]


def _targets_value(args, value, name: str, truncate: bool):
    """``(*targets, value[, truncate])`` or ``(sequence, value[, truncate])``."""
    args = list(args)
    if args and _is_seq(args[0]):
        targets, rest = list(args[0]), args[1:]
        if rest and isinstance(rest[-1], bool):
            truncate = rest.pop()
        if value is None:
            if not rest:
                raise TypeError(f"missing required argument: {name!r}")
            value = rest[-1]
        return [int(t) for t in targets], value, truncate
    if value is None:
        if len(args) >= 2 and isinstance(args[-1], bool):
            truncate = args.pop()
        if not args:
            raise TypeError(f"missing required argument: {name!r}")
        return [int(t) for t in args[:-1]], args[-1], truncate
    return [int(t) for t in args], value, truncate


def _u32(targets: list[int]):
    arr = (ctypes.c_uint32 * max(1, len(targets)))(*targets)
    return arr, len(targets)


class PauliSum:
    """A weighted sum of Pauli strings on the GPU (see the module docstring).

    Attributes mirror the reference dataclass: ``initial_terms``, ``n_qubits``,
    ``coefficients``, ``min_abs_coeff`` (default 1e-10), ``max_pauli_weight`` (None = no cap),
    ``preserve_strings``.  Extra keyword-only options: ``clifford_angles`` (treat rotations
    at +-pi/2 as the Clifford they equal), ``exact_order`` (keep the reference's term order
    through every op; disables fused rotation runs, which give the same terms and coefficients
    in another order), ``device`` (CUDA ordinal), ``capacity`` (initial term capacity).
    """

    def __init__(self, initial_terms: Sequence[str], n_qubits: int, coefficients: Sequence[float] = (),
                 min_abs_coeff: float = 1e-10, max_pauli_weight: int | None = None,
                 max_loss_weight: int | None = None, preserve_strings: Sequence[str] | None = None,
                 *, clifford_angles: bool = False, exact_order: bool = False, device: int = 0,
                 capacity: int = 0):
        if not initial_terms:
            raise ValueError("At least one term must be provided to initialize PauliSum.")
        for term in initial_terms:
            if len(term) != n_qubits:
                raise ValueError("All terms must have the same length! Expected length "
                                 f"{n_qubits}, but got term of length {len(term)}: {term!r}")
        if not coefficients:
            coefficients = (1.0,) * len(initial_terms)
        if len(coefficients) != len(initial_terms):
            raise ValueError("Initial terms and coefficients need to be of same length!")
        self.initial_terms = list(initial_terms)
        self.n_qubits = int(n_qubits)
        self.coefficients = tuple(float(c) for c in coefficients)
        self.min_abs_coeff = float(min_abs_coeff)
        self.max_pauli_weight = max_pauli_weight
        # the plain tiers accept max_loss_weight and ignore it, as the reference's binding does
        # (crates/ppvm-python-native/src/interface.rs:89); LossyPauliSum applies it
        self.max_loss_weight = max_loss_weight
        self.preserve_strings = list(preserve_strings) if preserve_strings else None
        self.W = G.lossy_words(self.n_qubits) if self._LOSSY else G.words(self.n_qubits)
        self._h = ctypes.c_void_p()
        mw = UMAX if max_pauli_weight is None else int(max_pauli_weight)
        flags = (FLAG_CLIFFORD_ANGLES if clifford_angles else 0) | (FLAG_EXACT_ORDER if exact_order else 0)
        flags |= FLAG_LOSSY if self._LOSSY else 0
        self._check(lib().ppvm_sum_create2(ctypes.byref(self._h), self.n_qubits, self.min_abs_coeff, mw,
                                           int(capacity), flags, int(device)))
        if self._LOSSY and max_loss_weight is not None:
            self._check(lib().ppvm_sum_set_max_loss_weight(self._h, int(max_loss_weight)))
        if self.preserve_strings:
            for s in self.preserve_strings:
                if len(s) != n_qubits:
                    raise ValueError("All preserve strings must have length n_qubits "
                                     f"({n_qubits}); got {len(s)}: {s!r}")
            px, pz = self._planes(self.preserve_strings)
            self._check(lib().ppvm_sum_set_preserve(self._h, _p64(px), _p64(pz), len(self.preserve_strings)))
        x, z = self._planes(self.initial_terms)
        c = np.asarray(self.coefficients, dtype=np.float64)
        self._check(lib().ppvm_sum_add_terms(self._h, _p64(x), _p64(z), _pd(c), len(c)))

    # ---- construction helpers --------------------------------------------------------------
    @classmethod
    def new(cls, n_qubits: int, terms, min_abs_coeff: float = 1e-10, max_pauli_weight: int | None = None,
            max_loss_weight: int | None = None, preserve_strings: Sequence[str] | None = None, **kw):
        """As ``ppvm.PauliSum.new``: ``"IX"``, compact ``"X1"``, or ``(str, coeff)`` terms."""
        if isinstance(terms, (str, tuple)):
            terms = [terms]
        parsed = [_parse_term(t, n_qubits) for t in terms]
        return cls([s for s, _ in parsed], n_qubits, [c for _, c in parsed], min_abs_coeff,
                   max_pauli_weight, max_loss_weight, preserve_strings, **kw)

    @staticmethod
    def _check(status: int):
        if status == OK:
            return
        msg = lib().ppvm_last_error_string().decode(errors="replace")
        if status == EINVAL:
            raise ValueError(msg)
        raise PPVMError(status, msg)

    _LOSSY = False  # LossyPauliSum: words over I, X, Y, Z and L

    def _parse(self, w):
        return G.parse_lossy_word(w, self.n_qubits) if self._LOSSY else G.parse_word(w, self.n_qubits)

    def _word(self, x, z) -> str:
        return G.lossy_word_str(x, z, self.n_qubits) if self._LOSSY else G.word_str(x, z, self.n_qubits)

    def _planes(self, words):
        x = np.zeros((len(words), self.W), dtype=np.uint64)
        z = np.zeros((len(words), self.W), dtype=np.uint64)
        for i, w in enumerate(words):
            x[i], z[i] = self._parse(w)
        return x, z

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            try:
                lib().ppvm_sum_destroy(h)
            except Exception:
                pass
            self._h = None

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._h

    # ---- size / copies ---------------------------------------------------------------------
    def __len__(self) -> int:
        n = ctypes.c_size_t()
        self._check(lib().ppvm_len(self._h, ctypes.byref(n)))
        return n.value

    def __copy__(self) -> "PauliSum":
        new = object.__new__(type(self))
        new.__dict__.update({k: v for k, v in self.__dict__.items() if k != "_h"})
        new._h = ctypes.c_void_p()
        self._check(lib().ppvm_sum_clone(self._h, ctypes.byref(new._h)))
        return new

    def copy(self) -> "PauliSum":
        return self.__copy__()

    def __eq__(self, other) -> bool:
        if not isinstance(other, PauliSum):
            return NotImplemented
        out = ctypes.c_int()
        self._check(lib().ppvm_equal(self._h, other._h, ctypes.byref(out)))
        return bool(out.value)

    __hash__ = None

    # ---- readout ------------------------------------------------------------------------------
    def export(self):
        """(x[N, W], z[N, W], c[N]) numpy arrays in the sum's iteration order."""
        n = len(self)
        x = np.zeros((max(n, 1), self.W), dtype=np.uint64)
        z = np.zeros((max(n, 1), self.W), dtype=np.uint64)
        c = np.zeros(max(n, 1), dtype=np.float64)
        got = ctypes.c_size_t()
        self._check(lib().ppvm_export_terms(self._h, _p64(x), _p64(z), _pd(c), n, ctypes.byref(got)))
        return x[: got.value], z[: got.value], c[: got.value]

    @property
    def terms(self) -> list[tuple[str, float]]:
        x, z, c = self.export()
        return [(self._word(x[i], z[i]), float(c[i])) for i in range(len(c))]

    def weights(self) -> list[tuple[str, int]]:
        x, z, _ = self.export()
        n = len(x)
        w = np.zeros(max(n, 1), dtype=np.uint32)
        got = ctypes.c_size_t()
        self._check(lib().ppvm_weights(self._h, w.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), n,
                                       ctypes.byref(got)))
        return [(self._word(x[i], z[i]), int(w[i])) for i in range(got.value)]

    def current_max_weight(self) -> int:
        out = ctypes.c_uint64()
        self._check(lib().ppvm_current_max_weight(self._h, ctypes.byref(out)))
        return int(out.value)

    def overlap_with_zero(self) -> float:
        out = ctypes.c_double()
        self._check(lib().ppvm_overlap_with_zero(self._h, ctypes.byref(out)))
        return out.value

    expectation = overlap_with_zero

    def overlap(self, other: "PauliSum") -> float:
        """sum_k self[k] * other[k] (tr(A^dag B) in the Pauli basis)."""
        out = ctypes.c_double()
        self._check(lib().ppvm_overlap(self._h, other._h, ctypes.byref(out)))
        return out.value

    def trace(self, pattern: str) -> float:
        out = ctypes.c_double()
        self._check(lib().ppvm_trace(self._h, pattern.encode(), ctypes.byref(out)))
        return out.value

    def __str__(self) -> str:
        # Display (crates/ppvm-pauli-sum/src/sum/display.rs:29-45): stable sort by weight.
        ts = self.terms
        ts = sorted(ts, key=lambda t: sum(ch != "I" for ch in t[0]))
        return " + ".join(f"{c:.3f} * {w}" for w, c in ts)

    def __repr__(self) -> str:
        return f"PauliSum({self})"

    def truncate(self) -> None:
        self._check(lib().ppvm_truncate(self._h))

    # ---- gates ----------------------------------------------------------------------------------
    def _g1(self, fn, targets, truncate):
        arr, k = _u32(_targets(targets))
        self._check(fn(self._h, arr, k, int(bool(truncate))))

    def x(self, *t, truncate: bool = True): self._g1(lib().ppvm_x, t, truncate)
    def y(self, *t, truncate: bool = True): self._g1(lib().ppvm_y, t, truncate)
    def z(self, *t, truncate: bool = True): self._g1(lib().ppvm_z, t, truncate)
    def h(self, *t, truncate: bool = True): self._g1(lib().ppvm_h, t, truncate)
    def s(self, *t, truncate: bool = True): self._g1(lib().ppvm_s, t, truncate)
    def s_dag(self, *t, truncate: bool = True): self._g1(lib().ppvm_s_dag, t, truncate)
    def sqrt_x(self, *t, truncate: bool = True): self._g1(lib().ppvm_sqrt_x, t, truncate)
    def sqrt_x_dag(self, *t, truncate: bool = True): self._g1(lib().ppvm_sqrt_x_dag, t, truncate)
    def sqrt_y(self, *t, truncate: bool = True): self._g1(lib().ppvm_sqrt_y, t, truncate)
    def sqrt_y_dag(self, *t, truncate: bool = True): self._g1(lib().ppvm_sqrt_y_dag, t, truncate)
    def cnot(self, *t, truncate: bool = True): self._g1(lib().ppvm_cnot, t, truncate)
    def cz(self, *t, truncate: bool = True): self._g1(lib().ppvm_cz, t, truncate)
    def cy(self, *t, truncate: bool = True): self._g1(lib().ppvm_cy, t, truncate)
    cx = zcx = cnot
    zcz = cz
    zcy = cy

    def _rot(self, fn, args, theta, truncate):
        targets, theta, truncate = _targets_value(args, theta, "theta", truncate)
        arr, k = _u32(targets)
        self._check(fn(self._h, arr, k, float(theta), int(bool(truncate))))

    def rx(self, *a, theta=None, truncate: bool = True): self._rot(lib().ppvm_rx, a, theta, truncate)
    def ry(self, *a, theta=None, truncate: bool = True): self._rot(lib().ppvm_ry, a, theta, truncate)
    def rz(self, *a, theta=None, truncate: bool = True): self._rot(lib().ppvm_rz, a, theta, truncate)
    def rxx(self, *a, theta=None, truncate: bool = True): self._rot(lib().ppvm_rxx, a, theta, truncate)
    def ryy(self, *a, theta=None, truncate: bool = True): self._rot(lib().ppvm_ryy, a, theta, truncate)
    def rzz(self, *a, theta=None, truncate: bool = True): self._rot(lib().ppvm_rzz, a, theta, truncate)

    def r(self, addr0: int, axis_angle: float, theta: float, truncate: bool = True) -> None:
        """R(phi, theta) = RZ(phi) RX(theta) RZ(-phi), emitted in Heisenberg order."""
        self._check(lib().ppvm_r(self._h, int(addr0), float(axis_angle), float(theta), int(bool(truncate))))

    def pauli_rotation(self, pauli: str, theta: float, truncate: bool = True) -> None:
        """exp(-i theta/2 P) for a Pauli string P of length n (or compact, e.g. "X0Z3")."""
        word, _ = _parse_term(pauli, self.n_qubits)
        gx, gz = G.parse_word(word, self.n_qubits)
        if self._LOSSY:  # the generator has no loss bits: the upper words stay 0
            gx = np.concatenate([gx, np.zeros_like(gx)])
            gz = np.concatenate([gz, np.zeros_like(gz)])
        self._check(lib().ppvm_pauli_rotation(self._h, _p64(gx), _p64(gz), float(theta), int(bool(truncate))))

    # ---- noise (diagonal channels) --------------------------------------------------------------
    def pauli_error(self, *a, p=None, truncate: bool = True):
        targets, p, truncate = _targets_value(a, p, "p", truncate)
        arr, k = _u32(targets)
        pp = (ctypes.c_double * 3)(*[float(v) for v in p])
        self._check(lib().ppvm_pauli_error(self._h, arr, k, pp, int(bool(truncate))))

    def x_error(self, *a, p=None, truncate: bool = True):
        targets, p, truncate = _targets_value(a, p, "p", truncate)
        self.pauli_error(targets, p=[p, 0.0, 0.0], truncate=truncate)

    def y_error(self, *a, p=None, truncate: bool = True):
        targets, p, truncate = _targets_value(a, p, "p", truncate)
        self.pauli_error(targets, p=[0.0, p, 0.0], truncate=truncate)

    def z_error(self, *a, p=None, truncate: bool = True):
        targets, p, truncate = _targets_value(a, p, "p", truncate)
        self.pauli_error(targets, p=[0.0, 0.0, p], truncate=truncate)

    def depolarize1(self, *a, p=None, truncate: bool = True):
        targets, p, truncate = _targets_value(a, p, "p", truncate)
        arr, k = _u32(targets)
        self._check(lib().ppvm_depolarize1(self._h, arr, k, float(p), int(bool(truncate))))

    def depolarize2(self, *a, p=None, truncate: bool = True):
        targets, p, truncate = _targets_value(a, p, "p", truncate)
        arr, k = _u32(targets)
        self._check(lib().ppvm_depolarize2(self._h, arr, k, float(p), int(bool(truncate))))

    def two_qubit_pauli_error(self, *a, p=None, truncate: bool = True):
        """``two_qubit_pauli_error(targets, p, truncate=True)``: flat pair list, 15
        probabilities of IX IY IZ XI XX XY XZ YI YX YY YZ ZI ZX ZY ZZ (noise.rs:39-105)."""
        targets, p, truncate = _targets_value(a, p, "p", truncate)
        pv = [float(v) for v in p]
        if len(pv) != 15:
            raise ValueError("two_qubit_pauli_error needs 15 probabilities")
        arr, k = _u32(targets)
        pp = (ctypes.c_double * 15)(*pv)
        self._check(lib().ppvm_two_qubit_pauli_error(self._h, arr, k, pp, int(bool(truncate))))

    def amplitude_damping(self, addr0: int, gamma: float, truncate: bool = True):
        """Amplitude damping of qubit ``addr0`` (noise.rs:132-163): Z -> (1-g) Z + g I,
        X/Y -> sqrt(1-g) X/Y."""
        if int(addr0) < 0:
            raise ValueError("qubit index out of range")
        self._check(lib().ppvm_amplitude_damping(self._h, int(addr0), float(gamma), int(bool(truncate))))

    # ---- gate lists ------------------------------------------------------------------------------
    def run(self, ops) -> None:
        """Runs a gate list (``ppvm_b200.gates`` tuples, or a ``GateList`` built once with
        ``ops_array``) in one device submission."""
        gl = ops if isinstance(ops, GateList) else ops_array(ops)
        self._check(lib().ppvm_gate_list_run(self._h, gl.ptr, len(gl)))

    def truncate_budget(self, budget: int, net=None, lattice: int = 0, layers_left: int = 0,
                        digit_bits: int = 8) -> None:
        """Keeps the ``budget`` terms of highest priority, in order: |c| (``net`` None) or the
        score of a ``TermPriorityNet`` (ppvm_b200.learned) on an ``lattice`` x ``lattice`` grid
        with ``layers_left`` layers still to apply."""
        self._check(lib().ppvm_truncate_budget(self._h, int(budget), net._h if net is not None else None,
                                               int(lattice), int(layers_left), int(digit_bits)))

    def features(self, lattice: int, layers_left: int) -> np.ndarray:
        """Per-term features of learned truncation, ``[len(self), 8]`` float32, iteration order."""
        n = len(self)
        out = np.zeros((max(n, 1), 8), dtype=np.float32)
        got = ctypes.c_size_t()
        self._check(lib().ppvm_term_features(self._h, int(lattice), int(layers_left),
                                             out.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), n,
                                             ctypes.byref(got)))
        return out[: got.value]

    def launch_count(self) -> int:
        """Kernels this sum has launched since it was created."""
        n = ctypes.c_uint64()
        self._check(lib().ppvm_launch_count(self._h, ctypes.byref(n)))
        return int(n.value)

    def transfer_counters(self) -> tuple[int, int]:
        """Bytes copied host->device and device->host by this sum since it was created."""
        h2d, d2h = ctypes.c_uint64(), ctypes.c_uint64()
        self._check(lib().ppvm_transfer_counters(self._h, ctypes.byref(h2d), ctypes.byref(d2h)))
        return int(h2d.value), int(d2h.value)

    def live_counts(self) -> np.ndarray:
        """Live terms entering each op of the last ``run`` (term-gate-updates numerator)."""
        n = ctypes.c_size_t()
        self._check(lib().ppvm_last_run_live_counts(self._h, None, 0, ctypes.byref(n)))
        out = np.zeros(max(n.value, 1), dtype=np.uint64)
        self._check(lib().ppvm_last_run_live_counts(self._h, _p64(out), n.value, ctypes.byref(n)))
        return out[: n.value]

    def profile(self, on: bool = True) -> None:
        self._check(lib().ppvm_profile_enable(self._h, int(on)))

    def profile_read(self) -> dict[str, dict[str, float]]:
        cap = 16
        names = ctypes.create_string_buffer(512)
        ms = (ctypes.c_double * cap)()
        ln = (ctypes.c_uint64 * cap)()
        by = (ctypes.c_uint64 * cap)()
        n = ctypes.c_size_t()
        self._check(lib().ppvm_profile_read(self._h, names, 512, ms, ln, by, cap, ctypes.byref(n)))
        labels = names.raw.split(b"\0")[: n.value]
        return {labels[i].decode(): {"ms": ms[i], "launches": int(ln[i]), "bytes": int(by[i])}
                for i in range(n.value)}

    def set_stream(self, stream_handle: int | None) -> None:
        """Binds the sum to an existing cudaStream_t (e.g. torch.cuda.current_stream().cuda_stream)."""
        self._check(lib().ppvm_sum_set_stream(self._h, ctypes.c_void_p(stream_handle or 0)))


OP_DTYPE = np.dtype([("code", "<u4"), ("q0", "<u4"), ("q1", "<u4"), ("flags", "<u4"),
                     ("theta", "<f8"), ("p", "<f8", (3,))])
assert OP_DTYPE.itemsize == ctypes.sizeof(Op)


class LossyPauliSum(PauliSum):
    """A PauliSum of lossy words: each qubit is I, X, Y, Z or L (lost), as the reference's
    ``ppvm.LossyPauliSum`` (ppvm-python/src/ppvm/paulisum.py:419-499) over LossyPauliWord
    (crates/ppvm-pauli-word/src/loss/data.rs).  ``max_loss_weight`` caps the number of L per
    term at truncation.  At most 256 qubits.  The loss channels take the reference's
    arguments; gates treat L as the reference does (a lost qubit is left alone)."""

    _LOSSY = True

    def loss_channel(self, addr0: int, p: float, *, truncate: bool = True) -> None:
        """L -> L + p I on ``addr0``; I, X, Y, Z -> (1 - p) (noise.rs:165-181)."""
        arr, k = _u32([int(addr0)])
        self._check(lib().ppvm_loss_channel(self._h, arr, k, float(p), int(bool(truncate))))

    def correlated_loss_channel(self, addr0: int, addr1: int, p, *, truncate: bool = True) -> None:
        """Correlated loss of the pair (noise.rs:184-243); p = (both, one, second after first)."""
        pv = [float(v) for v in p]
        if len(pv) != 3:
            raise ValueError("correlated_loss_channel needs 3 probabilities")
        arr, k = _u32([int(addr0), int(addr1)])
        self._check(lib().ppvm_correlated_loss_channel(self._h, arr, k, (ctypes.c_double * 3)(*pv),
                                                       int(bool(truncate))))

    def reset_loss_channel(self, addr0: int, *, truncate: bool = True) -> None:
        """L -> 0 on ``addr0``; I, Z -> themselves + L (noise.rs:245-275)."""
        arr, k = _u32([int(addr0)])
        self._check(lib().ppvm_reset_loss_channel(self._h, arr, k, int(bool(truncate))))


class GateList:
    """A gate list packed as ``ppvm_op`` records (numpy-backed), ready for the C ABI."""

    def __init__(self, arr: np.ndarray):
        self.arr = arr
        self.ptr = arr.ctypes.data_as(ctypes.POINTER(Op))

    def __len__(self) -> int:
        return len(self.arr)


def ops_array(ops) -> GateList:
    """Packs ``(code, q0, q1, theta, (p0, p1, p2))`` tuples into ``ppvm_op`` records."""
    arr = np.zeros(max(1, len(ops)), dtype=OP_DTYPE)
    if ops:
        code, q0, q1, theta, p = zip(*ops)
        arr["code"][: len(ops)] = code
        arr["q0"][: len(ops)] = q0
        arr["q1"][: len(ops)] = q1
        arr["theta"][: len(ops)] = theta
        arr["p"][: len(ops)] = p
    return GateList(arr[: len(ops)] if ops else arr[:0])


def clifford_tableau(n_qubits: int, ops):
    """Images of X_q (row 2q) and Z_q (row 2q+1) under a list of Clifford ops, as the engine
    composes them (host only): ``(img_x[2n, W], img_z[2n, W], sign[2n])``, image =
    (-1)^sign * word.  Rotations at +-pi/2 count as the Clifford they equal."""
    W = G.words(n_qubits)
    gl = ops_array(ops)
    ix = np.zeros((2 * n_qubits, W), dtype=np.uint64)
    iz = np.zeros((2 * n_qubits, W), dtype=np.uint64)
    sg = np.zeros(2 * n_qubits, dtype=np.uint8)
    st = lib().ppvm_clifford_tableau(n_qubits, gl.ptr, len(gl), _p64(ix), _p64(iz),
                                     sg.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)))
    if st != OK:
        msg = lib().ppvm_last_error_string().decode(errors="replace")
        raise ValueError(msg) if st == EINVAL else PPVMError(st, msg)
    return ix, iz, sg


def _p64(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))


def _pd(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


__all__ = ["PauliSum", "PPVMError", "GateList", "ops_array", "clifford_tableau"]
