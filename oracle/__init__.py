"""CPU oracle for the ADGA ladder hot path (test infrastructure only).

This package restates the reference's per-(q, omega) ladder loop in plain
NumPy/SciPy (``adga_oracle``) and in C (``adga_oracle.c``, the timed CPU
baseline).  It is a checker: only ``tests/``, ``__graft_entry__.smoke()`` and
the ``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` may import or
run it.  The product path (``adga_b200``) never calls into this package.

Parity status: the reference Fortran cannot be compiled in this image (no
gfortran, no LAPACK/HDF5/MPI), so parity with the Fortran binary itself is
UNPINNED except where the reference ships a data file: ``create_u`` is pinned
against ``documentation/examples/umatrix`` and the ``.hk`` reader against
``srvo3-testdata/srvo3_k20.hk`` (both checked in ``tests/test_oracle.py``).
All other routines are pinned by analytic known-answer tests only.
"""
