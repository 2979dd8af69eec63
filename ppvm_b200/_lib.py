"""ctypes binding of libppvm_cuda.so (the C ABI of include/ppvm_cuda.h).

The library is the only compute path: there is no CPU fallback.  If it is missing or
cannot be loaded, ``lib()`` raises immediately.
"""

from __future__ import annotations

import ctypes
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libppvm_cuda.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "ppvm_cuda.h")

OK, EINVAL, ECAPACITY, ECUDA, ETIMEOUT, ENODEV = range(6)
FLAG_CLIFFORD_ANGLES = 1
FLAG_EXACT_ORDER = 2
FLAG_LOSSY = 4
UMAX = (1 << 64) - 1


class PPVMError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"ppvm status {status}: {msg}")
        self.status = status


class Op(ctypes.Structure):
    """``ppvm_op``."""

    _fields_ = [
        ("code", ctypes.c_uint32),
        ("q0", ctypes.c_uint32),
        ("q1", ctypes.c_uint32),
        ("flags", ctypes.c_uint32),
        ("theta", ctypes.c_double),
        ("p", ctypes.c_double * 3),
    ]


_P = ctypes.c_void_p
_U32P = ctypes.POINTER(ctypes.c_uint32)
_U64P = ctypes.POINTER(ctypes.c_uint64)
_DP = ctypes.POINTER(ctypes.c_double)
_SZ = ctypes.c_size_t
_SZP = ctypes.POINTER(ctypes.c_size_t)
_I = ctypes.c_int

_SIGS = {
    "ppvm_sum_create": [ctypes.POINTER(_P), ctypes.c_uint32, ctypes.c_double, ctypes.c_uint64, _SZ],
    "ppvm_sum_create2": [ctypes.POINTER(_P), ctypes.c_uint32, ctypes.c_double, ctypes.c_uint64, _SZ,
                         ctypes.c_uint32, _I],
    "ppvm_sum_destroy": [_P],
    "ppvm_sum_clone": [_P, ctypes.POINTER(_P)],
    "ppvm_sum_set_stream": [_P, _P],
    "ppvm_sum_add_terms": [_P, _U64P, _U64P, _DP, _SZ],
    "ppvm_sum_add_string": [_P, ctypes.c_char_p, ctypes.c_double],
    "ppvm_sum_set_preserve": [_P, _U64P, _U64P, _SZ],
    "ppvm_len": [_P, _SZP],
    "ppvm_export_terms": [_P, _U64P, _U64P, _DP, _SZ, _SZP],
    "ppvm_weights": [_P, _U32P, _SZ, _SZP],
    "ppvm_current_max_weight": [_P, _U64P],
    "ppvm_equal": [_P, _P, ctypes.POINTER(_I)],
    "ppvm_r": [_P, ctypes.c_uint32, ctypes.c_double, ctypes.c_double, _I],
    "ppvm_pauli_rotation": [_P, _U64P, _U64P, ctypes.c_double, _I],
    "ppvm_pauli_error": [_P, _U32P, _SZ, _DP, _I],
    "ppvm_depolarize1": [_P, _U32P, _SZ, ctypes.c_double, _I],
    "ppvm_depolarize2": [_P, _U32P, _SZ, ctypes.c_double, _I],
    "ppvm_loss_channel": [_P, _U32P, _SZ, ctypes.c_double, _I],
    "ppvm_reset_loss_channel": [_P, _U32P, _SZ, _I],
    "ppvm_correlated_loss_channel": [_P, _U32P, _SZ, ctypes.POINTER(ctypes.c_double), _I],
    "ppvm_sum_set_max_loss_weight": [_P, ctypes.c_uint64],
    "ppvm_two_qubit_pauli_error": [_P, _U32P, _SZ, _DP, _I],
    "ppvm_amplitude_damping": [_P, ctypes.c_uint32, ctypes.c_double, _I],
    "ppvm_truncate": [_P],
    "ppvm_overlap_with_zero": [_P, _DP],
    "ppvm_expectation": [_P, _DP],
    "ppvm_trace": [_P, ctypes.c_char_p, _DP],
    "ppvm_overlap": [_P, _P, _DP],
    "ppvm_gate_list_run": [_P, ctypes.POINTER(Op), _SZ],
    "ppvm_last_run_live_counts": [_P, _U64P, _SZ, _SZP],
    "ppvm_clifford_tableau": [ctypes.c_uint32, ctypes.POINTER(Op), _SZ, _U64P, _U64P,
                              ctypes.POINTER(ctypes.c_uint8)],
    "ppvm_transfer_counters": [_P, _U64P, _U64P],
    "ppvm_launch_count": [_P, _U64P],
    "ppvm_truncate_budget": [_P, ctypes.c_uint64, _P, ctypes.c_uint32, ctypes.c_uint32, _I],
    "ppvm_term_features": [_P, ctypes.c_uint32, ctypes.c_uint32, ctypes.POINTER(ctypes.c_float), _SZ, _SZP],
    "ppvm_mlp_create": [ctypes.POINTER(_P), ctypes.c_uint64, _I],
    "ppvm_mlp_destroy": [_P],
    "ppvm_mlp_set_params": [_P, ctypes.POINTER(ctypes.c_float), _SZ],
    "ppvm_mlp_get_params": [_P, ctypes.POINTER(ctypes.c_float), _SZ],
    "ppvm_mlp_train": [_P, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float), _SZ, _I, _I,
                       ctypes.c_float, ctypes.c_uint64, ctypes.POINTER(ctypes.c_float)],
    "ppvm_mlp_grad": [_P, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float), _SZ,
                      ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float)],
    "ppvm_mlp_predict": [_P, ctypes.POINTER(ctypes.c_float), _SZ, ctypes.POINTER(ctypes.c_float)],
    "ppvm_sum_shard_export": [_P, _U64P, _U64P, ctypes.c_uint32, _P, _SZ, _U64P],
    "ppvm_sum_shard_append": [_P, _P, _SZ],
    "ppvm_batch_create": [ctypes.POINTER(_P), _SZ, _U32P, _DP, _U64P, ctypes.c_uint32, _I],
    "ppvm_batch_destroy": [_P],
    "ppvm_batch_set_stream": [_P, _P],
    "ppvm_batch_add_terms": [_P, _SZ, _U64P, _U64P, _DP, _SZ],
    "ppvm_batch_set_ops": [_P, _SZ, ctypes.POINTER(Op), _SZ],
    "ppvm_batch_set_ops_all": [_P, ctypes.POINTER(ctypes.POINTER(Op)), _SZP],
    "ppvm_batch_run": [_P],
    "ppvm_batch_run_persistent": [_P],
    "ppvm_batch_reserve": [_P, _U64P],
    "ppvm_batch_get_capacity": [_P, _U64P],
    "ppvm_batch_set_config": [_P, _I, _I, _I],
    "ppvm_batch_get_config": [_P, ctypes.POINTER(_I), ctypes.POINTER(_I), ctypes.POINTER(_I)],
    "ppvm_batch_autotune": [_P, ctypes.POINTER(_I), ctypes.POINTER(_I), ctypes.POINTER(_I), _DP],
    "ppvm_batch_overlap_with_zero": [_P, _DP],
    "ppvm_batch_len": [_P, _SZ, _SZP],
    "ppvm_batch_export_terms": [_P, _SZ, _U64P, _U64P, _DP, _SZ, _SZP],
    "ppvm_batch_term_gate_updates": [_P, _U64P, _U64P],
    "ppvm_batch_transfer_counters": [_P, _U64P, _U64P],
    "ppvm_release_cached_memory": [],
    "ppvm_profile_enable": [_P, _I],
    "ppvm_profile_read": [_P, ctypes.c_char_p, _SZ, _DP, _U64P, _U64P, _SZ, _SZP],
}
for _g in ("x", "y", "z", "h", "s", "s_dag", "sqrt_x", "sqrt_x_dag", "sqrt_y", "sqrt_y_dag",
           "cnot", "cz", "cy"):
    _SIGS[f"ppvm_{_g}"] = [_P, _U32P, _SZ, _I]
for _g in ("rx", "ry", "rz", "rxx", "ryy", "rzz"):
    _SIGS[f"ppvm_{_g}"] = [_P, _U32P, _SZ, ctypes.c_double, _I]

_lib = None


def header_functions() -> list[str]:
    """Names of the functions include/ppvm_cuda.h declares."""
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(ppvm_[a-z0-9_]+)\s*\(", text)))


def lib() -> ctypes.CDLL:
    """Loads the CUDA library once; raises if it is absent."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python ppvm_b200/build.py` "
                              "(there is no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        for name, args in _SIGS.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = ctypes.c_int
        L.ppvm_last_error_string.restype = ctypes.c_char_p
        L.ppvm_last_error_string.argtypes = []
        L.ppvm_version.restype = ctypes.c_char_p
        L.ppvm_version.argtypes = []
        _lib = L
    return _lib


def check(status: int) -> None:
    if status != OK:
        raise PPVMError(status, lib().ppvm_last_error_string().decode(errors="replace"))
