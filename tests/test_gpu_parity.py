"""GPU parity of the C-ABI path against the FP64 oracle.

Tolerances (normwise max-abs relative error against the oracle):
  FP64 path  <= 1e-10   (the reference's own FP64 bar)
  mixed path <= 1e-8    (FP32/BF16x3 LU + FP64 refinement)
"""
import dataclasses
from functools import lru_cache

import numpy as np
import pytest
from scipy.linalg import lapack

import adga_b200
from adga_b200 import Ladder, run_ladder, synth
from oracle import adga_oracle as O
from tests.helpers import oracle_run, problem, qw_points, rel_err, to_inputs

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-10, "mixed": 1e-8}
KEYS = ["chi_dens", "chi_magn", "bubble_nl", "chi_loc_dens", "chi_loc_magn", "sigma",
        "sigma_dmft", "bubble_loc", "chi_qw_dens", "chi_qw_magn"]


def compare(got, want, tol, keys=KEYS):
    errs = {k: rel_err(got[k], want[k]) for k in keys}
    bad = {k: v for k, v in errs.items() if not v <= tol}
    assert not bad, f"parity failed: {bad} (all: {errs})"
    return errs


@pytest.mark.parametrize("name", ["t1", "t2", "t3", "t5", "t3m"])
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_full_ladder_matches_oracle(name, prec):
    p = problem(name)
    got = run_ladder(p, prec)
    want = oracle_run(p)
    assert np.all(got["status"] >= 0)
    compare(got, want, TOL[prec])
    if prec == "mixed":
        # the mixed LU must converge on its own (no FP64 re-solve)
        assert got["stats"]["mixed_fallbacks"] == 0
        assert got["stats"]["max_refine_iters"] <= 4


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_c0_slice_matches_oracle(prec):
    """single-orbital simple-cubic workload, one bosonic slice plus the next
    omega's first points (crossing an omega boundary mid-batch)."""
    p = problem("c0")
    s = p.spec
    qs, qe = 10 * s.nqp + 1, 11 * s.nqp + 7          # omega = 0 slice, then omega = 1
    got = run_ladder(p, prec, qwstart=qs, qwstop=qe)
    want = oracle_run(p, qwstart=qs, qwstop=qe)
    compare(got, want, TOL[prec])


@lru_cache(maxsize=None)
def _c0_full_grid_oracle():
    return oracle_run(problem("c0"))


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_c0_full_grid_matches_oracle(prec):
    """The whole single-orbital simple-cubic workload: 125 q x 21 omega =
    2625 points (BSE N = 40), every output against the oracle, the mixed
    path without FP64 re-solves."""
    p = problem("c0")
    got = run_ladder(p, prec)
    want = _c0_full_grid_oracle()
    assert got["status"].shape == (2625,) and np.all(got["status"] == 0)
    compare(got, want, TOL[prec])
    if prec == "mixed":
        assert got["stats"]["mixed_fallbacks"] == 0


def test_partial_range_starting_mid_omega():
    """A block that starts mid-slice adds no local terms for that omega
    (the reference only adds them where the block holds iq = 1)."""
    p = problem("t3")
    s = p.spec
    qs, qe = 2, s.nqp * 2 + 1
    got = run_ladder(p, "fp64", qwstart=qs, qwstop=qe)
    want = oracle_run(p, qwstart=qs, qwstop=qe)
    compare(got, want, TOL["fp64"])


def test_big_box_bubble_option():
    p = problem("t2")
    got = run_ladder(p, "fp64", bubble_big_box=True)
    want = oracle_run(p, bubble_big_box=True)
    compare(got, want, TOL["fp64"])


def test_chi_only_and_eom_only():
    p = problem("t2")
    got = run_ladder(p, "fp64", do_eom=False)
    want = oracle_run(p, do_eom=False)
    compare(got, want, TOL["fp64"], ["chi_dens", "chi_magn", "bubble_nl"])
    assert np.max(np.abs(got["sigma_nl"])) == 0
    got = run_ladder(p, "fp64", do_chi=False)
    want = oracle_run(p, do_chi=False)
    compare(got, want, TOL["fp64"], ["sigma", "sigma_dmft"])


def test_zero_bosonic_box():
    spec = dataclasses.replace(synth.SPECS["t3"], name="t3w0", iwb=0)
    p = synth.make_problem(spec)
    got = run_ladder(p, "fp64")
    want = oracle_run(p)
    compare(got, want, TOL["fp64"])


# ---- per-routine entry points ---------------------------------------------------
@pytest.fixture(scope="module")
def lad_t3():
    p = problem("t3")
    lad = Ladder.from_problem(p)
    for iwb in range(-p.spec.iwb, p.spec.iwb + 1):
        lad.set_vertex(iwb, *p.vertex(iwb))
    yield p, lad
    lad.close()


def test_chi0_loc_routines(lad_t3):
    p, lad = lad_t3
    o = O.Oracle(to_inputs(p))
    for iwf, iwb in [(-3, 1), (0, 0), (2, -1)]:
        np.testing.assert_allclose(np.diag(lad.get_chi0_loc(iwf, iwb)), o.get_chi0_loc(iwf, iwb),
                                   rtol=1e-14)
        np.testing.assert_allclose(np.diag(lad.get_chi0_loc_inv(iwf, iwb)),
                                   o.get_chi0_loc_inv(iwf, iwb), rtol=1e-14)


def test_chi0_q_routine(lad_t3):
    p, lad = lad_t3
    o = O.Oracle(to_inputs(p))
    s = p.spec
    for iq, iwb in [(1, 0), (2, 1), (2, -1)]:
        c, b = lad.chi0_q(iq, iwb)
        want = np.stack([o.chi0_q(iq - 1, nu, iwb) for nu in range(-s.iwf, s.iwf)], axis=2)
        assert rel_err(c, want) < 1e-13
        scratch = {k: np.zeros((p.ndim2, p.ndim2, 2 * s.iwb + 1), complex)
                   for k in ("bubble_loc", "chi_loc_dens", "chi_loc_magn")}
        loc = o.local_block(iwb, 1, scratch)
        bw = want.sum(axis=2) / p.beta ** 2 - loc[2]
        assert rel_err(b, bw) < 1e-12


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_bse_point_routine(lad_t3, prec):
    p, lad = lad_t3
    o = O.Oracle(to_inputs(p))
    scratch = {k: np.zeros((p.ndim2, p.ndim2, 2 * p.spec.iwb + 1), complex)
               for k in ("bubble_loc", "chi_loc_dens", "chi_loc_magn")}
    for iq, iwb in [(1, 0), (2, 1)]:
        loc = o.local_block(iwb, 0, scratch)
        res = o.point(iq - 1, iwb, loc)
        ed, em, gq, info = lad.bse_point(iq, iwb, prec)
        assert info == 0
        assert rel_err(ed, res["etaqd"]) < TOL[prec]
        assert rel_err(em, res["etaqm"]) < TOL[prec]
        assert rel_err(gq, res["gammaqd"]) < 1e-12


def test_gamma_w_and_calc_chi_qw(lad_t3):
    p, lad = lad_t3
    o = O.Oracle(to_inputs(p))
    scratch = {k: np.zeros((p.ndim2, p.ndim2, 2 * p.spec.iwb + 1), complex)
               for k in ("bubble_loc", "chi_loc_dens", "chi_loc_magn")}
    loc = o.local_block(1, 0, scratch)
    gd, gm = lad.get_gamma_w(1)
    assert rel_err(gd, loc[5]) < 1e-12 and rel_err(gm, loc[6]) < 1e-12
    rng = np.random.default_rng(3)
    chi = np.asfortranarray(rng.normal(size=(p.ndim2, p.ndim2)) + 0j)
    c0 = rng.normal(size=(p.ndim2, p.ndim2, 2 * p.spec.iwf)) + 1j * rng.normal(size=(p.ndim2, p.ndim2, 2 * p.spec.iwf))
    want = chi.copy()
    o.calc_chi_qw(want, gd, c0)
    lad.calc_chi_qw(chi, gd, c0)
    assert rel_err(chi, want) < 1e-13


def test_eom_routines(lad_t3):
    p, lad = lad_t3
    s = p.spec
    o = O.Oracle(to_inputs(p))
    scratch = {k: np.zeros((p.ndim2, p.ndim2, 2 * s.iwb + 1), complex)
               for k in ("bubble_loc", "chi_loc_dens", "chi_loc_magn")}
    loc = o.local_block(0, 0, scratch)
    res = o.point(1, 0, loc)
    rng = np.random.default_rng(5)
    sig0 = rng.normal(size=(p.ndim, p.ndim, 2 * s.iwf, s.nkp)) * (1 + 0j)
    want = np.asfortranarray(sig0.copy())
    o.calc_eom_dynamic(res["etaqd"], res["etaqm"], res["gammaqd"], 0, 1, want)
    got = np.asfortranarray(sig0.copy())
    lad.calc_eom_dynamic(res["etaqd"], res["etaqm"], res["gammaqd"], 0, 2, got)
    assert rel_err(got, want) < 1e-12
    sd = np.zeros((p.ndim, p.ndim, 2 * s.iwf), complex, order="F")
    wd = sd.copy()
    o.calc_eom_static(0, wd)
    o.calc_eom_dmft(loc[5], 0, wd)
    lad.calc_eom_static(1, sd)
    lad.calc_eom_dmft(loc[5], 0, sd)
    assert rel_err(sd, wd) < 1e-13


def test_inverse_matrix_gpu():
    rng = np.random.default_rng(7)
    for n in (1, 3, 40, 100, 257):
        A = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n)) + n ** 0.5 * np.eye(n)
        inv, ierr, erstr = adga_b200.inverse_matrix(A)
        want, info, _ = O.inverse_matrix(A)
        assert ierr == 0 and erstr == ""
        assert rel_err(inv, want) < 1e-11
    S = np.zeros((5, 5), complex)
    S[0, 0] = 1
    _, ierr, erstr = adga_b200.inverse_matrix(S)
    assert ierr == 2 and erstr == "ERROR in ZGETRF"


def test_index_kq_gpu():
    nk = (4, 6, 2)
    q = O.generate_q_vol(nk, (2, 3, 1))
    np.testing.assert_array_equal(adga_b200.index_kq(nk, q), O.index_kq(nk, q))
    ks = np.array([1, 7, 48, 13], dtype=np.int32)
    np.testing.assert_array_equal(adga_b200.index_kq(nk, q, ks), O.index_kq(nk, q, ks))


def test_set_vertex_required():
    p = problem("t2")
    lad = Ladder.from_problem(p)
    try:
        with pytest.raises(adga_b200.AdgaError):
            lad.ladder_run(1, 2, "fp64")
    finally:
        lad.close()
