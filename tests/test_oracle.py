"""CPU tests of the oracle: golden vectors of the reference and analytic
known-answer tests of the ladder algebra."""
import os
from pathlib import Path

import numpy as np
import pytest
from scipy.linalg import lapack

from adga_b200 import synth
from oracle import adga_oracle as O
from tests.helpers import oracle_run, problem, rel_err, to_inputs

GOLD = Path(__file__).resolve().parent / "golden"
# the reference checkout (read-only); its data-file test is skipped where it is absent
REF = Path(os.environ.get("ADGA_REFERENCE", "/root/reference"))


# ---- golden vectors from the reference's data files -----------------------
def test_create_u_matches_reference_umatrix():
    g = np.load(GOLD / "umatrix_example.npz")
    Umat, u, ut = O.create_u([(3, 0)], [5.0], [3.5], [0.75])
    np.testing.assert_array_equal(Umat, g["Umat"])
    # compound forms follow from the same tensor
    for i in range(3):
        for j in range(3):
            for k in range(3):
                for l in range(3):
                    assert u[i * 3 + k, l * 3 + j] == g["Umat"][i, j, k, l]
                    assert ut[i * 3 + k, l * 3 + j] == g["Umat"][i, j, l, k]


def test_synthetic_kanamori_matches_create_u():
    for nd, U, V, J in [(1, 2.0, 2.0, 0.0), (2, 4.0, 2.8, 0.6), (3, 5.0, 3.5, 0.75), (5, 3.0, 2.0, 0.5)]:
        Um_o, u_o, ut_o = O.create_u([(nd, 0)], [U], [V], [J])
        Um_s = synth.kanamori_umat(nd, U, V, J)
        np.testing.assert_array_equal(Um_o, Um_s)
        u_s, ut_s = synth.compound_u(Um_s)
        np.testing.assert_array_equal(u_o, u_s)
        np.testing.assert_array_equal(ut_o, ut_s)


@pytest.mark.skipif(not (REF / "srvo3-testdata/srvo3_k20.hk").exists(), reason="reference data absent")
def test_read_hk_matches_digest():
    g = np.load(GOLD / "srvo3_hk_digest.npz")
    kd, hk = O.read_hk(REF / "srvo3-testdata/srvo3_k20.hk")
    assert hk.shape == (int(g["ndim"]), int(g["ndim"]), int(g["nkp"]))
    pick = g["kpick"]
    np.testing.assert_allclose(kd[:, pick].T, g["k_data"], rtol=0, atol=0)
    np.testing.assert_allclose(np.transpose(hk[:, :, pick], (2, 0, 1)), g["hk_pick"], rtol=0, atol=0)
    assert abs(hk.sum() - g["hk_sum"]) < 1e-9 * abs(g["hk_sum"])
    # the .hk k ordering is kz fastest (src/kq_tools.f90:119-144)
    np.testing.assert_allclose(kd, synth.k_points((20, 20, 20)), atol=1e-12)


# ---- k-q tools ---------------------------------------------------------------
def test_k_minus_q_brute_force():
    nk = (4, 6, 2)
    for ik in range(1, 49):
        for iq in range(1, 49):
            kx, ky, kz = O.k_vector(ik, nk)
            qx, qy, qz = O.k_vector(iq, nk)
            want = O.k_index((kx - qx) % 4, (ky - qy) % 6, (kz - qz) % 2, nk)
            assert O.k_minus_q(ik, iq, nk) == want


def test_generate_q_vol_subset():
    q = O.generate_q_vol((20, 20, 20), (10, 10, 10))
    assert len(q) == 1000 and q[0] == 1
    kx, ky, kz = O.k_vector(q, (20, 20, 20))
    assert np.all(kx % 2 == 0) and np.all(ky % 2 == 0) and np.all(kz % 2 == 0)


# ---- small inverses ----------------------------------------------------------
def test_closed_form_inverses_vs_lapack():
    rng = np.random.default_rng(0)
    for n, f in [(2, O.inverse_matrix_2), (3, O.inverse_matrix_3)]:
        A = rng.normal(size=(50, n, n)) + 1j * rng.normal(size=(50, n, n)) + 3 * np.eye(n)
        B = f(A)
        for a, b in zip(A, B):
            inv, info, _ = O.inverse_matrix(a)
            assert info == 0
            np.testing.assert_allclose(b, inv, rtol=1e-12, atol=1e-13)


def test_inverse_matrix_reports_singular():
    A = np.zeros((4, 4), complex)
    A[0, 0] = 1
    _, info, erstr = O.inverse_matrix(A)
    assert info == 2 and erstr == "ERROR in ZGETRF"


# ---- known-answer tests of the ladder algebra ----------------------------------
def test_zero_vertex():
    """chi_loc = chi0_loc: F~ = 0, gamma = 0, A = 1, eta = 0, so
    chi(q,w) = bubble_nl + bubble_loc and Sigma_nl = 0."""
    p = problem("t2")

    def vtx(iwb):
        d = np.diag(synth.chi0_loc_diag(p, iwb))
        return d, d.copy()

    out = oracle_run(p, vertex=vtx)
    s = p.spec
    widx = out["qw"][:, 0] + s.iwb
    want = out["bubble_nl"] + out["bubble_loc"][:, :, widx]
    assert rel_err(out["chi_dens"], want) < 1e-13
    assert rel_err(out["chi_magn"], want) < 1e-13
    assert np.max(np.abs(out["sigma_nl"])) < 1e-12 * np.max(np.abs(p.siw))


def test_flat_band_is_local():
    """H(k) = const and G_imp = lattice G: chi0^q = chi0^w, bubble_nl = 0 and
    chi(q, w) = chi_loc(w) for every q."""
    import dataclasses
    p = synth.make_problem(dataclasses.replace(synth.SPECS["t2"], offdiag=0.0))
    p.hk[:] = p.hk[:, :, :1]
    inp0 = to_inputs(p)
    o = O.Oracle(inp0)
    for n in range(-p.iwmax, p.iwmax):
        g = o.gk(n)[0]
        p.giw[n + p.iwmax] = np.diag(g)
    # only valid with an orbital-diagonal H
    assert np.allclose(p.hk[0, 1], 0)
    p._vcache.clear()
    out = oracle_run(p)
    s = p.spec
    assert np.max(np.abs(out["bubble_nl"])) < 1e-12 * np.max(np.abs(out["bubble_loc"]))
    widx = out["qw"][:, 0] + s.iwb
    assert rel_err(out["chi_dens"], out["chi_loc_dens"][:, :, widx]) < 1e-10
    assert rel_err(out["chi_magn"], out["chi_loc_magn"][:, :, widx]) < 1e-10


def test_single_orbital_gamma_form():
    """ndim = 1: the reference's F~-form ladder equals the Gamma-form BSE
    chi_q = (chi0_q^-1 + Gamma)^-1 with Gamma = chi_loc^-1 - chi0_loc^-1, summed
    over nu, nu' / beta^2 -- an independent dense computation."""
    p = problem("t1")
    s = p.spec
    out = oracle_run(p)
    inp = to_inputs(p)
    o = O.Oracle(inp)
    for n, (iwb, iq) in enumerate(out["qw"]):
        cd, cm = p.vertex(int(iwb))
        c0l = synth.chi0_loc_diag(p, int(iwb))
        c0q = np.array([o.chi0_q(int(iq), nu, int(iwb))[0, 0] for nu in range(-s.iwf, s.iwf)])
        for ch, chi in ((0, cd), (1, cm)):
            sym = 0.5 * (chi + chi.T)
            Gam = np.linalg.inv(sym) - np.diag(1 / c0l)
            chiq = np.linalg.inv(np.diag(1 / c0q) + Gam)
            want = chiq.sum() / p.beta ** 2
            got = (out["chi_dens"] if ch == 0 else out["chi_magn"])[0, 0, n]
            assert abs(got - want) < 1e-10 * abs(want), (n, ch, got, want)


def test_sigma_mirror_symmetry():
    p = problem("t3")
    out = oracle_run(p)
    sig = out["sigma_nl"]
    iwf = p.spec.iwf
    for nu in range(iwf):
        np.testing.assert_array_equal(sig[:, :, iwf - 1 - nu, :],
                                      np.conj(np.transpose(sig[:, :, iwf + nu, :], (1, 0, 2))))


def test_local_chi_symmetrisation_is_transpose_average():
    p = problem("t2")
    inp = to_inputs(p)
    o = O.Oracle(inp)
    N = p.maxdim
    scratch = {k: np.zeros((p.ndim2, p.ndim2, 2 * p.spec.iwb + 1), complex)
               for k in ("bubble_loc", "chi_loc_dens", "chi_loc_magn")}
    loc = o.local_block(0, 0, scratch)
    Fd = loc[3]
    c0inv = loc[0].T.reshape(-1)
    chi = (Fd + np.eye(N)) / c0inv[None, :]
    np.testing.assert_allclose(chi, chi.T, rtol=1e-12, atol=1e-14 * np.abs(chi).max())


@pytest.mark.parametrize("name", ["t2", "t3"])
def test_multi_orbital_gamma_form(name):
    """Orbital compound indices: chi(q,w)[i1,i2] = beta^-2 sum_{nu,nu'}
    [(chi0_q^-1 + Gamma)^-1][(i1,nu),(i2,nu')] with chi0_q block-diagonal in nu
    and Gamma = sym(chi_loc)^-1 - chi0_loc^-1."""
    p = problem(name)
    s = p.spec
    out = oracle_run(p)
    o = O.Oracle(to_inputs(p))
    nd2, N = p.ndim2, p.maxdim
    for n in range(0, len(out["qw"]), max(1, len(out["qw"]) // 5)):
        iwb, iq = (int(x) for x in out["qw"][n])
        c0l = synth.chi0_loc_diag(p, iwb)
        blk = np.zeros((N, N), complex)
        for dum, nu in enumerate(range(-s.iwf, s.iwf)):
            blk[dum * nd2:(dum + 1) * nd2, dum * nd2:(dum + 1) * nd2] = o.chi0_q(iq, nu, iwb)
        for ch, chi in enumerate(p.vertex(iwb)):
            sym = 0.5 * (chi + chi.T)
            Gam = np.linalg.inv(sym) - np.diag(1 / c0l)
            chiq = np.linalg.inv(np.linalg.inv(blk) + Gam)
            want = chiq.reshape(2 * s.iwf, nd2, 2 * s.iwf, nd2).sum(axis=(0, 2)) / p.beta ** 2
            got = (out["chi_dens"] if ch == 0 else out["chi_magn"])[:, :, n]
            assert rel_err(got, want) < 1e-10, (name, n, ch)
