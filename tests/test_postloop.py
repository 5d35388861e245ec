"""Post-loop assembly (src/main.F90:869-890): add_siw_dmft, get_sigma_g_loc, get_ndga.

CPU: the oracle restatement against known answers -- with a zero non-local
self-energy, gloc is the k-mean of the DMFT lattice Green's function built in
accumulate_chi0 (src/one_particle_quant_module.f90:240-271) and obeys
G(-nu-1) = G(nu)^dagger; n_dga_k is real with 1/2 added on the diagonal.
GPU (through the C ABI): adga_post_loop on a handle's own Sigma_nl after a full
FP64 ladder, and on a caller-supplied Sigma (also on an EOM k subset), against
the oracle to 1e-12.
"""
import numpy as np
import pytest

from adga_b200 import Ladder
from adga_b200.ladder import generate_q_vol
from oracle import adga_oracle as O
from tests.helpers import oracle_run, problem, rel_err, to_inputs

TOL = 1e-12


def test_oracle_post_loop_zero_sigma_is_dmft_lattice():
    p = problem("t2")
    inp = to_inputs(p)
    s = p.spec
    nd, iwf = s.ndim, s.iwf
    out = O.post_loop(inp, np.zeros((nd, nd, 2 * iwf, inp.nkp), complex))
    orc = O.Oracle(inp)
    for n in (0, 1, iwf, inp.iwmax - 1):
        g = orc.gk(n).mean(axis=0)                  # (nd, nd) mean over k
        assert rel_err(out["gloc"][n + inp.iwmax], g) < 1e-13
        assert rel_err(out["gloc"][-n - 1 + inp.iwmax], g.conj().T) < 1e-13
    assert np.allclose(out["sigma_loc"][0, 0, :], p.siw[np.arange(-iwf, iwf) + inp.iwmax, 0])
    assert np.all(out["n_dga_k"].imag == 0)
    assert np.allclose(out["n_dga"], [out["n_dga_k"][:, i, i].mean() for i in range(nd)])


@pytest.mark.gpu
def test_post_loop_after_ladder_matches_oracle():
    p = problem("t3")
    inp = to_inputs(p)
    want_run = oracle_run(p)
    want = O.post_loop(inp, want_run["sigma_nl"])
    with Ladder.from_problem(p) as lad:
        for iwb in range(-p.spec.iwb, p.spec.iwb + 1):
            lad.set_vertex(iwb, *p.vertex(iwb))
        lad.ladder_run(1, None, "fp64")
        got = lad.post_loop()                       # the handle's own Sigma_nl
        sig_nl = lad.get_outputs()["sigma_nl"]
        got2 = lad.post_loop(sigma_sum=sig_nl)      # the same Sigma from the caller
    for k in ("sigma_loc", "gloc", "n_dga_k", "n_dga"):
        assert rel_err(got[k], want[k]) < 1e-10, (k, rel_err(got[k], want[k]))
        assert rel_err(got2[k], got[k]) < TOL, k
    assert rel_err(got2["sigma_sum"], want["sigma_sum"]) < 1e-10


@pytest.mark.gpu
def test_post_loop_on_eom_k_subset():
    p = problem("t2")
    s = p.spec
    inp = to_inputs(p)
    kdata = np.array([1, 3, 4, 7, inp.nkp], dtype=np.int32)
    rng = np.random.default_rng(3)
    sig = (rng.standard_normal((s.ndim, s.ndim, 2 * s.iwf, len(kdata))) +
           1j * rng.standard_normal((s.ndim, s.ndim, 2 * s.iwf, len(kdata)))) * 0.05
    want = O.post_loop(inp, sig, k_data_eom=kdata)
    lad = Ladder(ndim=s.ndim, nk=s.nk, nq=s.nq, iwmax=p.iwmax, iwfmax_small=s.iwf, iwbmax_small=s.iwb,
                 beta=p.beta, mu=p.mu, iw_data=p.iw_data, hk=p.hk, siw=p.siw, giw=p.giw, dc=p.dc,
                 u=p.u, u_tilde=p.u_tilde, n_dmft=p.n_dmft, q_data=generate_q_vol(s.nk, s.nq),
                 k_data_eom=kdata)
    try:
        got = lad.post_loop(sigma_sum=sig, want=("n_dga_k", "n_dga"))
        for k in ("sigma_sum", "n_dga_k", "n_dga"):
            assert rel_err(got[k], want[k]) < TOL, (k, rel_err(got[k], want[k]))
        with pytest.raises(Exception):
            lad.post_loop(sigma_sum=sig, want=("gloc",))   # needs the full k mesh
    finally:
        lad.close()
