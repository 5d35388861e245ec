"""Transform path of the chi0 bubble and the EOM (k_dft.cu): the cyclic k-sums
through DFTs of the G table, folded onto the q mesh, against the direct
k - q kernels and the oracle.

ADGA_DFT_MIN_POINTS=1 forces the transform for every batch, ADGA_BUBBLE=direct
keeps the direct kernels; both are read when a handle is created.
"""
import numpy as np
import pytest

from adga_b200 import Ladder, synth
from adga_b200.ladder import generate_q_vol
from tests.helpers import library_env as env, oracle_run, problem, rel_err

pytestmark = pytest.mark.gpu
TRANSFORM = {"ADGA_DFT_MIN_POINTS": "1"}
DIRECT = {"ADGA_BUBBLE": "direct"}
OUT_KEYS = ("chi_qw_dens", "chi_qw_magn", "bubble_nl", "sigma_nl", "chi_loc_dens", "chi_loc_magn", "sigma_dmft")


def make_ladder(p, settings, q_data=None, k_data_eom=None, bubble_big_box=False):
    s = p.spec
    with env(settings):
        lad = Ladder(ndim=s.ndim, nk=s.nk, nq=s.nq, iwmax=p.iwmax, iwfmax_small=s.iwf, iwbmax_small=s.iwb,
                     beta=p.beta, mu=p.mu, iw_data=p.iw_data, hk=p.hk, siw=p.siw, giw=p.giw, dc=p.dc,
                     u=p.u, u_tilde=p.u_tilde, n_dmft=p.n_dmft,
                     q_data=generate_q_vol(s.nk, s.nq) if q_data is None else q_data,
                     k_data_eom=k_data_eom, bubble_big_box=bubble_big_box)
    for iwb in range(-s.iwb, s.iwb + 1):
        lad.set_vertex(iwb, *p.vertex(iwb))
    return lad


def run(p, settings, prec="fp64", **kw):
    lad = make_ladder(p, settings, **kw)
    try:
        nqw = lad.nqp * (2 * p.spec.iwb + 1)
        lad.ladder_run(1, nqw, prec)
        out = lad.get_outputs()
        out.update(lad.assemble(out, p.siw))
        return out
    finally:
        lad.close()


@pytest.mark.parametrize("name", ["t1", "t2", "t3", "t5"])
def test_transform_matches_oracle(name):
    p = problem(name)
    got = run(p, TRANSFORM)
    want = oracle_run(p)
    for k in ("chi_dens", "chi_magn", "sigma"):
        assert rel_err(got[k], want[k]) < 1e-10, (k, rel_err(got[k], want[k]))


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_transform_matches_direct(prec):
    """The mixed path agrees with itself to its refinement tolerance (its last
    correction, bounded by 1e-10 max|X|, may be left unapplied)."""
    p = problem("t3b")
    a, b = run(p, TRANSFORM, prec), run(p, DIRECT, prec)
    tol = 1e-12 if prec == "fp64" else 1e-9
    for k in OUT_KEYS:
        assert rel_err(a[k], b[k]) < tol, (k, rel_err(a[k], b[k]))


def test_transform_on_an_irregular_q_list():
    """q points that are not a sub-mesh: the fold mesh is the whole k mesh."""
    p = problem("t2")
    q = np.array([1, 6, 11, 30], dtype=np.int32)        # nqp = 4 points of the 4x4x2 mesh
    a, b = run(p, TRANSFORM, q_data=q), run(p, DIRECT, q_data=q)
    for k in OUT_KEYS:
        assert rel_err(a[k], b[k]) < 1e-12, (k, rel_err(a[k], b[k]))


def test_transform_eom_on_a_k_subset():
    p = problem("t3b")
    kdata = np.array([1, 5, 17, 40, 100, 216], dtype=np.int32)
    full = run(p, TRANSFORM)
    a, b = run(p, TRANSFORM, k_data_eom=kdata), run(p, DIRECT, k_data_eom=kdata)
    assert rel_err(a["sigma_nl"], b["sigma_nl"]) < 1e-12
    assert rel_err(a["sigma_nl"], full["sigma_nl"][..., kdata - 1]) < 1e-12


def test_transform_big_box_bubble():
    p = problem("t2")
    a = run(p, TRANSFORM, bubble_big_box=True)
    b = run(p, DIRECT, bubble_big_box=True)
    for k in OUT_KEYS:
        assert rel_err(a[k], b[k]) < 1e-12, (k, rel_err(a[k], b[k]))


@pytest.mark.parametrize("par", ["t", "U"])
def test_transform_tangents_match_direct(par):
    p = problem("t2")
    dhk, du, dut, dvertex = synth.tangent_inputs(p, par)
    res = []
    for settings in (TRANSFORM, DIRECT):
        lad = make_ladder(p, settings)
        try:
            for iwb in range(-p.spec.iwb, p.spec.iwb + 1):
                if dvertex is not None:
                    lad.set_vertex_tangent(iwb, *dvertex(iwb))
            lad.set_tangent(dhk, du, dut)
            lad.ladder_run_tangent()
            res.append(lad.get_tangent_outputs())
        finally:
            lad.close()
    for k in OUT_KEYS:
        assert rel_err(res[0][k], res[1][k]) < 1e-12, (k, rel_err(res[0][k], res[1][k]))
