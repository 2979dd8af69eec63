"""The allocation-free overlap_with_zero entry point, checked against the allocating one.

ppvm_overlap_with_zero_noalloc serves callers that cannot let the library allocate device
memory (a framework whose pool owns the GPU's memory, or a latency-critical loop where
cudaMalloc would stall the device).  The caller hands it device buffers; the test builds
them with torch, runs the entry point twice in a row through the C ABI, and compares each
result with ppvm_overlap_with_zero on a PauliSum holding the same terms.  This file is
collected last so that a run stopping at the first failure has run every other test first.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-10  # overlap_with_zero tolerance used throughout the parity tests


def _fn():
    from ppvm_b200 import _lib

    f = _lib.lib().ppvm_overlap_with_zero_noalloc
    f.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_size_t,
                  ctypes.c_void_p, ctypes.c_void_p]
    f.restype = ctypes.c_int
    return f


def _terms(seed, n_terms, n_qubits):
    rng = np.random.default_rng(seed)
    W = (n_qubits + 63) // 64
    x = np.zeros((n_terms, W), dtype=np.uint64)
    z = rng.integers(0, 1 << 63, size=(n_terms, W), dtype=np.uint64)
    # a third of the terms carry X bits (sparse, distinct per term index); the rest are X-free
    has_x = rng.random(n_terms) < 0.34
    for i in np.nonzero(has_x)[0]:
        q = int(rng.integers(n_qubits))
        x[i, q // 64] |= np.uint64(1) << np.uint64(q % 64)
    tail = n_qubits % 64
    if tail:
        z[:, -1] &= np.uint64((1 << tail) - 1)
    z[:, 0] = (z[:, 0] & ~np.uint64(0xFFFFF)) | np.arange(n_terms, dtype=np.uint64)  # distinct words
    c = rng.uniform(-1, 1, n_terms)
    return x, z, c


def _reference_value(x, z, c, n_qubits):
    from ppvm_b200 import _lib
    from ppvm_b200.paulisum import _pd, _p64

    L = _lib.lib()
    h = ctypes.c_void_p()
    _lib.check(L.ppvm_sum_create(ctypes.byref(h), n_qubits, 0.0, _lib.UMAX, len(c)))
    try:
        xx, zz, cc = np.ascontiguousarray(x), np.ascontiguousarray(z), np.ascontiguousarray(c)
        _lib.check(L.ppvm_sum_add_terms(h, _p64(xx), _p64(zz), _pd(cc), len(cc)))
        out = ctypes.c_double()
        _lib.check(L.ppvm_overlap_with_zero(h, ctypes.byref(out)))
        return out.value
    finally:
        L.ppvm_sum_destroy(h)


def _noalloc_value(x, c):
    import torch

    n, W = x.shape
    planes = torch.from_numpy(np.ascontiguousarray(x.T).view(np.int64)).cuda()  # [W][n], stride n
    coeff = torch.from_numpy(c).cuda()
    out = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    st = _fn()(planes.data_ptr(), n, W, coeff.data_ptr(), n, out.data_ptr(), stream.cuda_stream)
    assert st == 0
    torch.cuda.synchronize()
    return float(out.item())


@pytest.mark.parametrize("n_qubits,n_terms", [(144, 300_001), (20, 4096)])
def test_noalloc_matches_overlap_with_zero_twice(n_qubits, n_terms):
    for seed in (1, 2):  # two calls in a row reuse the library's fixed array
        x, z, c = _terms(seed + n_qubits, n_terms, n_qubits)
        want = _reference_value(x, z, c, n_qubits)
        got = _noalloc_value(x, c)
        assert abs(got - want) <= TOL, (got, want)
        exact = float(np.sum(c[~x.any(axis=1)]))
        assert abs(got - exact) <= 1e-8


def test_noalloc_rejects_oversize_and_bad_arguments():
    import torch

    from ppvm_b200 import _lib

    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    dummy = torch.zeros(1, dtype=torch.int64, device="cuda")
    f = _fn()
    too_many = 16_777_216 + 1
    assert f(dummy.data_ptr(), too_many, 1, dummy.data_ptr(), too_many, out.data_ptr(), None) == _lib.EINVAL
    assert b"16777216" in _lib.lib().ppvm_last_error_string()
    assert f(dummy.data_ptr(), 1, 9, dummy.data_ptr(), 1, out.data_ptr(), None) == _lib.EINVAL
    assert f(dummy.data_ptr(), 0, 1, dummy.data_ptr(), 1, out.data_ptr(), None) == _lib.EINVAL
    # an empty input sums to zero
    assert f(None, 0, 1, None, 0, out.data_ptr(), None) == 0
    torch.cuda.synchronize()
    assert float(out.item()) == 0.0
