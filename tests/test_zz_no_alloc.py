"""The allocation-free inverse entry point (adga_inverse_matrix_z_noalloc).

It serves callers that cannot call cudaMalloc -- their device memory belongs
to another allocator, or the library must not grow the device footprint --
so it takes caller-owned device buffers and keeps all LU scratch in a static
device array (n <= ADGA_NOALLOC_MAX_N).  These tests drive it through the C
ABI on device buffers owned by torch:

* calls in a row (the shared scratch keeps the previous call's contents),
  including the largest size n = ADGA_NOALLOC_MAX_N, each checked against the
  FP64 oracle's zgetrf + zgetri inverse and against the allocating entry
  point adga_inverse_matrix_z;
* a singular matrix: the LAPACK-style info comes back as the return value
  and in ierr, equal to zgetrf's;
* a call on a non-default stream;
* no device memory is allocated by a call (free device memory unchanged);
* sizes beyond the limit are rejected.

The file name makes pytest collect it last.
"""
import ctypes as C

import numpy as np
import pytest

import adga_b200
from adga_b200 import _lib
from oracle.adga_oracle import inverse_matrix as oracle_inverse

pytestmark = pytest.mark.gpu
TOL = 1e-11
MAX_N = 256
ADGA_EINVAL = -1


def _matrix(rng, n):
    return rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n)) + np.sqrt(n) * np.eye(n)


def _to_device(A):
    import torch
    # column-major n x n on the device: A^T in row-major torch memory
    return torch.from_numpy(np.ascontiguousarray(A.T)).to("cuda")


def _call(dA, dI, n, ierr=None, stream=None):
    lib = _lib.load()
    return lib.adga_inverse_matrix_z_noalloc(C.c_void_p(dA.data_ptr()), C.c_void_p(dI.data_ptr()), n,
                                             C.byref(ierr) if ierr is not None else None,
                                             C.c_void_p(stream) if stream else None)


def _noalloc_inverse(A, stream=None):
    import torch
    n = A.shape[0]
    dA = _to_device(A)
    dI = torch.empty_like(dA)
    torch.cuda.synchronize()
    ierr = C.c_int(-99)
    rc = _call(dA, dI, n, ierr, stream)
    torch.cuda.synchronize()
    return rc, ierr.value, dI.cpu().numpy().T


def _rel(a, b):
    return np.max(np.abs(a - b)) / np.max(np.abs(b))


def test_noalloc_inverse_matches_oracle_and_allocating_entry_point_in_a_row():
    rng = np.random.default_rng(11)
    for n in (200, 37, MAX_N, 64):            # calls in a row, different sizes, the limit included
        A = _matrix(rng, n)
        rc, ierr, got = _noalloc_inverse(A)
        assert rc == 0 and ierr == 0, (n, rc, ierr)
        want, info, _ = oracle_inverse(A)
        assert info == 0
        assert _rel(got, want) < TOL, (n, _rel(got, want))
        alloc, ierr2, _ = adga_b200.inverse_matrix(A)
        assert ierr2 == 0
        assert _rel(got, alloc) < TOL, (n, _rel(got, alloc))


def test_noalloc_inverse_reports_singular_matrix_like_zgetrf():
    rng = np.random.default_rng(12)
    n = 96
    A = _matrix(rng, n)
    A[:, 70] = 0.0                            # exactly singular: zgetrf stops at column 71
    _, want_info, _ = oracle_inverse(A)
    assert want_info == 71
    rc, ierr, _ = _noalloc_inverse(A)
    assert ierr == want_info and rc == want_info
    # the info is returned also without an ierr pointer
    import torch
    dA = _to_device(A)
    dI = torch.empty_like(dA)
    assert _call(dA, dI, n) == want_info
    torch.cuda.synchronize()
    # and the next call on a regular matrix is clean again (info is cleared per call)
    B = _matrix(rng, n)
    rc, ierr, got = _noalloc_inverse(B)
    assert rc == 0 and ierr == 0
    assert _rel(got, oracle_inverse(B)[0]) < TOL


def test_noalloc_inverse_on_a_side_stream_allocates_nothing():
    import torch
    rng = np.random.default_rng(13)
    n = 160
    A = _matrix(rng, n)
    want = oracle_inverse(A)[0]
    s = torch.cuda.Stream()
    dA = _to_device(A)
    outs = [torch.empty_like(dA) for _ in range(3)]
    torch.cuda.synchronize()
    ierr = C.c_int(-99)
    assert _call(dA, outs[0], n, ierr, s.cuda_stream) == 0 and ierr.value == 0
    assert _call(dA, outs[1], n, ierr, s.cuda_stream) == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    assert _call(dA, outs[2], n, ierr, s.cuda_stream) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
    for o in outs:
        assert _rel(o.cpu().numpy().T, want) < TOL


def test_noalloc_inverse_rejects_oversize():
    import torch
    n = MAX_N + 1
    d = torch.zeros((n, n), dtype=torch.complex128, device="cuda")
    ierr = C.c_int(0)
    assert _call(d, d, n, ierr) == ADGA_EINVAL
