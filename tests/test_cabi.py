"""The C-ABI library loads and exports every symbol include/ppvm_cuda.h declares (no GPU)."""

import ctypes
import os
import subprocess

import pytest

from ppvm_b200 import _lib


def test_library_exports_every_header_symbol():
    L = _lib.lib()
    names = _lib.header_functions()
    assert len(names) > 40
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_no_device_is_reported_as_status():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    L = _lib.lib()
    h = ctypes.c_void_p()
    st = L.ppvm_sum_create(ctypes.byref(h), 4, 1e-10, _lib.UMAX, 0)
    assert st == _lib.ENODEV
    assert b"CUDA" in L.ppvm_last_error_string()


def test_op_struct_layout_matches_header():
    assert ctypes.sizeof(_lib.Op) == 4 * 4 + 8 + 3 * 8


def test_python_argument_forms():
    from ppvm_b200.paulisum import _targets, _targets_value

    assert _targets((0, 1, 2)) == [0, 1, 2]
    assert _targets(([0, 1],)) == [0, 1]
    assert _targets((range(3),)) == [0, 1, 2]
    assert _targets_value((0, 1, 0.5), None, "theta", True) == ([0, 1], 0.5, True)
    assert _targets_value(([0, 1], 0.5, False), None, "theta", True) == ([0, 1], 0.5, False)
    assert _targets_value((0, 1), 0.25, "theta", True) == ([0, 1], 0.25, True)
