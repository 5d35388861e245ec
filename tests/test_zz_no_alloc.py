"""The allocation-free inverse entry point (adga_inverse_matrix_z_noalloc).

It serves callers that cannot call cudaMalloc -- their device memory belongs
to another allocator, or the library must not grow the device footprint --
so it takes caller-owned device buffers and keeps all LU scratch in a static
device array (n <= ADGA_NOALLOC_MAX_N).  This test drives it through the C ABI
on device buffers owned by torch, twice in a row (the shared scratch keeps the
previous call's contents), and compares each result with the allocating
entry point adga_inverse_matrix_z within the tolerance of the other inverse
tests.  The file name makes pytest collect it last.
"""
import ctypes as C

import numpy as np
import pytest

import adga_b200
from adga_b200 import _lib

pytestmark = pytest.mark.gpu
TOL = 1e-11
MAX_N = 256


def _noalloc_inverse(A):
    import torch
    lib = _lib.load()
    n = A.shape[0]
    # column-major n x n on the device: store A^T in row-major torch memory
    dA = torch.from_numpy(np.ascontiguousarray(A.T)).to("cuda")
    dI = torch.empty_like(dA)
    torch.cuda.synchronize()
    ierr = C.c_int(-99)
    rc = lib.adga_inverse_matrix_z_noalloc(C.c_void_p(dA.data_ptr()), C.c_void_p(dI.data_ptr()), n,
                                           C.byref(ierr), None)
    torch.cuda.synchronize()
    return rc, ierr.value, dI.cpu().numpy().T


def test_noalloc_inverse_matches_allocating_entry_point_twice():
    rng = np.random.default_rng(11)
    for n in (200, 37):                       # two calls in a row, different sizes
        A = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n)) + np.sqrt(n) * np.eye(n)
        rc, ierr, got = _noalloc_inverse(A)
        assert rc == 0 and ierr == 0
        want, ierr2, _ = adga_b200.inverse_matrix(A)
        assert ierr2 == 0
        err = np.max(np.abs(got - want)) / np.max(np.abs(want))
        assert err < TOL, (n, err)


def test_noalloc_inverse_rejects_oversize():
    import torch
    lib = _lib.load()
    n = MAX_N + 1
    d = torch.zeros((n, n), dtype=torch.complex128, device="cuda")
    ierr = C.c_int(0)
    rc = lib.adga_inverse_matrix_z_noalloc(C.c_void_p(d.data_ptr()), C.c_void_p(d.data_ptr()), n,
                                           C.byref(ierr), None)
    assert rc == -1     # ADGA_EINVAL
