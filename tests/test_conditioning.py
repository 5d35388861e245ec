"""The ladder near a magnetic instability: ill-conditioned BSE matrices in a batch.

Near an instability the leading eigenvalue of the magnetic BSE kernel
chi0^q F~_m approaches 1 and 1 - chi0^q F~_m becomes nearly singular.  The
test model scales the local magnetic vertex of one bosonic frequency,
chi_loc_m' = chi0_loc + s (chi_loc_m - chi0_loc), so that F~_m' = s F~_m, with
s = (1 - delta) / mu* and mu* the largest-modulus eigenvalue of the kernel at
one chosen point: that point's magnetic matrix then has the eigenvalue delta
(condition number ~1e6 for delta = 1e-3, ~1e8 for 1e-5), its neighbours stay
moderately conditioned.  The whole slice runs as one batch:

* FP64 path: every output within C * eps * kappa of the oracle (kappa the
  largest condition number of the batch), the LAPACK-style status 0;
* mixed path: the FP32 factorisation cannot serve the worst point at
  kappa ~1e8, so its refinement must fail to converge and the point must be
  re-solved in FP64 (status -1, counted in mixed_fallbacks) while every other
  point stays on the mixed path; at kappa ~1e6 the point converges or falls
  back -- either way every output stays within the same bound.

An exactly singular BSE matrix (a zero pivot in exact arithmetic) cannot be
produced through the physical inputs, whose rounding never yields an exactly
zero column; the zero-pivot status path is covered on explicit matrices by
tests/test_gpu_parity.py and tests/test_zz_no_alloc.py.

Reference behaviour: inverse_matrix_z reports a zero pivot through ierr
(src/lapack_module.f90:52-56) and the loop stops on it (src/main.F90:734-737).
"""
import dataclasses
from functools import lru_cache

import numpy as np
import pytest

from adga_b200 import run_ladder, synth
from oracle.adga_oracle import Oracle
from tests.helpers import oracle_run, problem, rel_err, to_inputs

pytestmark = pytest.mark.gpu

EPS = 2.2e-16
IWB, IQ = 0, 3          # the point driven towards the instability (t3m, omega = 0 slice)


@lru_cache(maxsize=None)
def near_instability(name, delta):
    """(problem, kappa of every magnetic BSE matrix of the omega = IWB slice)."""
    p = problem(name)
    s = p.spec
    o = Oracle(to_inputs(p))
    scr = {k: np.zeros((p.ndim2, p.ndim2, 2 * s.iwb + 1), complex)
           for k in ("bubble_loc", "chi_loc_dens", "chi_loc_magn")}
    loc = o.local_block(IWB, IQ, scr)
    N = s.maxdim
    K = np.eye(N) - o.point(IQ, IWB, loc)["A_magn"]
    mu = np.linalg.eigvals(K)
    scale = (1.0 - delta) / mu[np.argmax(np.abs(mu))]
    chi_d, chi_m = p.vertex(IWB)
    c0 = np.diag(synth.chi0_loc_diag(p, IWB))
    chi_m2 = np.asfortranarray(c0 + scale * (0.5 * (chi_m + chi_m.T) - c0))
    p2 = dataclasses.replace(p, _vcache={})
    p2._vcache.update({w: p.vertex(w) for w in range(-s.iwb, s.iwb + 1)})
    p2._vcache[IWB] = (chi_d, chi_m2)
    o2 = Oracle(to_inputs(p2))
    loc2 = o2.local_block(IWB, 0, scr)
    kappa = [np.linalg.cond(o2.point(q, IWB, loc2)["A_magn"]) for q in range(s.nqp)]
    return p2, np.array(kappa)


def slice_range(p):
    s = p.spec
    q0 = (IWB + s.iwb) * s.nqp + 1
    return q0, q0 + s.nqp - 1


@pytest.mark.parametrize("delta", [1e-3, 1e-5])
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_near_instability_batch_matches_oracle(prec, delta):
    p, kappa = near_instability("t3m", delta)
    assert kappa[IQ] > (1e5 if delta == 1e-3 else 1e7), kappa
    assert np.argmax(kappa) == IQ
    qs, qe = slice_range(p)
    got = run_ladder(p, prec, qwstart=qs, qwstop=qe)
    want = oracle_run(p, qwstart=qs, qwstop=qe)
    st = got["stats"]
    tol = max(1e-10 if prec == "fp64" else 1e-8, 10 * EPS * kappa.max())
    for k in ("chi_dens", "chi_magn", "chi_qw_magn", "sigma", "bubble_nl"):
        assert rel_err(got[k], want[k]) <= tol, (k, rel_err(got[k], want[k]), tol)
    # the well-conditioned points alone meet the plain bar
    ok = [i for i in range(p.spec.nqp) if kappa[i] < 1e3]
    assert ok
    for k in ("chi_qw_dens", "chi_qw_magn"):
        err = rel_err(got[k][:, :, ok], want[k][:, :, ok])
        assert err <= (1e-10 if prec == "fp64" else 1e-8), (k, err)
    if prec == "fp64":
        assert np.all(got["status"] == 0) and st["mixed_fallbacks"] == 0
    else:
        fb = np.flatnonzero(got["status"] == -1)
        assert st["mixed_fallbacks"] == len(fb)
        assert np.all(got["status"][got["status"] != -1] == 0)
        # only ill-conditioned points leave the mixed path
        assert all(kappa[i] > 1e4 for i in fb), (fb, kappa)
        if delta == 1e-5:
            assert IQ in fb                     # kappa ~1e8: beyond the FP32 factors
