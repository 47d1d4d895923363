"""The allocation-free power iteration (pdfp_estimate_max_singular_value_noalloc).

Some callers cannot allocate device memory: a process whose HBM a framework
allocator reserved up front, where a fresh cudaMalloc fails or fragments the
pool, or a caller that must not trigger cudaFree's device-wide
synchronisation.  This entry point keeps its work vectors in a fixed 8 MiB
device array of the library instead.  The test allocates the caller's own
device arrays (the matrix) with torch, calls the entry point through the C
ABI twice in a row, and checks both results against the allocating entry
point pdfp_estimate_max_singular_value (same algorithm, start vector and
summation order; estimates within 1e-10 relative, equal iteration counts),
and two of the cases against the CPU oracle's power iteration as well.

It also checks that a call made after the first on a device changes neither
the device's free memory nor torch's allocator, runs a case near the scratch
limit (few iterations), and checks the host-side rejections.

This file sorts last so that a run stopping at the first failure has run
every other test before it.
"""
import ctypes as C

import numpy as np
import pytest
import scipy.sparse as sp

from pdfp_b200 import _lib as L
from pdfp_b200 import gpu

pytestmark = pytest.mark.gpu


def _device_csr(A):
    import torch
    A = sp.csr_matrix(A, dtype=np.float64)
    A.sort_indices()
    rp = torch.tensor(A.indptr.astype(np.int32), device="cuda")
    ci = torch.tensor(A.indices.astype(np.int32) if A.nnz else np.zeros(1, np.int32), device="cuda")
    v = torch.tensor(A.data if A.nnz else np.zeros(1), dtype=torch.float64, device="cuda")
    return rp, ci, v


def _ptr(t, ty):
    return C.cast(C.c_void_p(t.data_ptr()), C.POINTER(ty))


def _noalloc_on(m, n, a, at, max_iterations=5000, tolerance=1e-4):
    """One call of the entry point on device arrays a = (rp, ci, v) of A and at of A'."""
    import torch
    sigma = C.c_double()
    its = C.c_int32()
    torch.cuda.synchronize()
    rc = L.lib().pdfp_estimate_max_singular_value_noalloc(
        m, n, _ptr(a[0], C.c_int32), _ptr(a[1], C.c_int32), _ptr(a[2], C.c_double),
        _ptr(at[0], C.c_int32), _ptr(at[1], C.c_int32), _ptr(at[2], C.c_double),
        max_iterations, tolerance, None, C.byref(sigma), C.byref(its))
    L.check(rc)
    return sigma.value, its.value


def _device_pair(A):
    return _device_csr(A), _device_csr(sp.csr_matrix(A).T.tocsr())


def _noalloc(A, max_iterations=5000, tolerance=1e-4):
    m, n = A.shape
    a, at = _device_pair(A)
    return _noalloc_on(m, n, a, at, max_iterations, tolerance)


def _matrices():
    rng = np.random.default_rng(5)
    A1 = sp.random(300, 700, density=0.02, random_state=rng, format="csr")
    A2 = sp.random(2000, 3000, density=0.004, random_state=rng, format="csr")
    from pdfp_b200 import synthetic
    milp = synthetic.covering_p0201_like(1)
    return [A1, A2, milp.A]


@pytest.mark.parametrize("idx", [0, 1, 2])
def test_noalloc_matches_allocating_entry_point_twice(idx):
    A = _matrices()[idx]
    ref, ref_it = gpu.estimate_max_singular_value(A)
    for _ in range(2):  # the shared scratch keeps the previous call's contents
        s, it = _noalloc(A)
        assert s == pytest.approx(ref, rel=1e-10)
        assert it == ref_it


@pytest.mark.parametrize("idx", [0, 2])
def test_noalloc_matches_the_oracle(idx):
    """Pinned to the oracle's restatement of estimate_max_singular_value
    (src/preconditioner.jl:108-125) directly, not only through the allocating
    entry point: the same estimate to 1e-10 relative (the tolerance used against the
    allocating entry point) and the same iteration count."""
    from oracle import oracle as O
    A = _matrices()[idx]
    so, io = O.estimate_max_singular_value(sp.csr_matrix(A))
    s, it = _noalloc(A)
    assert s == pytest.approx(so, rel=1e-10)
    assert it == io


def test_noalloc_rejects_sizes_beyond_its_scratch():
    sigma = C.c_double()
    rc = L.lib().pdfp_estimate_max_singular_value_noalloc(
        600_000, 10, None, None, None, None, None, None, 10, 1e-4, None, C.byref(sigma), None)
    assert rc == L.E_UNSUPPORTED
    assert b"8 MiB" in L.lib().pdfp_last_error()


def test_noalloc_second_call_allocates_nothing():
    """After the first call on the device (which may commit the module's memory),
    a call leaves the device's free memory and torch's allocator unchanged."""
    import torch
    A = _matrices()[1]
    m, n = A.shape
    a, at = _device_pair(A)
    _noalloc_on(m, n, a, at)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    alloc0 = torch.cuda.memory_allocated()
    reserved0 = torch.cuda.memory_reserved()
    s, it = _noalloc_on(m, n, a, at)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    assert torch.cuda.memory_allocated() == alloc0
    assert torch.cuda.memory_reserved() == reserved0
    ref, ref_it = gpu.estimate_max_singular_value(A)
    assert s == pytest.approx(ref, rel=1e-10) and it == ref_it


def test_noalloc_near_its_size_limit():
    """2m + n + 2 = 1,047,002 of the 1,048,576 scratch values (the offsets of all three
    work vectors and the result near the end of the array), three iterations."""
    rng = np.random.default_rng(9)
    m, n = 349_000, 349_000
    A = sp.random(m, n, density=2.0 / n, random_state=rng, format="csr")
    ref, ref_it = gpu.estimate_max_singular_value(A, max_iterations=3)
    for _ in range(2):
        s, it = _noalloc(A, max_iterations=3)
        assert s == pytest.approx(ref, rel=1e-10)
        assert it == ref_it == 3


def test_noalloc_rejects_null_matrix_arrays():
    import torch
    A = _matrices()[0]
    m, n = A.shape
    a, at = _device_pair(A)
    sigma = C.c_double()
    torch.cuda.synchronize()
    rc = L.lib().pdfp_estimate_max_singular_value_noalloc(
        m, n, _ptr(a[0], C.c_int32), None, _ptr(a[2], C.c_double),
        _ptr(at[0], C.c_int32), _ptr(at[1], C.c_int32), _ptr(at[2], C.c_double),
        10, 1e-4, None, C.byref(sigma), None)
    assert rc == L.E_INVALID
    assert b"null matrix array" in L.lib().pdfp_last_error()
