"""Non-local interaction V(q) (do_vq): read_vq's index map, the density-channel
BSE term, the m_tot terms and calc_eom_static's Hartree/Fock parts
(src/main.F90:497-498,710-719; src/eom_module.f90:70-108,187-205;
src/interaction_module.f90:39-123).

CPU: the oracle's read_vq map against an einsum restatement.
GPU: full ladders with a seeded V(q) through the C ABI against the oracle run
with the same V(q): FP64 to 1e-10, mixed to 1e-8 (sigma_hf included).
"""
import dataclasses

import numpy as np
import pytest

from adga_b200 import Ladder
from oracle import adga_oracle as O
from tests.helpers import problem, qw_points, rel_err, to_inputs


def seeded_vq(nd, nqp, seed=11, scale=0.3):
    """V(q)_{ijkl}: density-density shape v_{ij}(q) delta_ik delta_jl, symmetric in
    (i, j), real, decaying with q, plus a small seeded general part."""
    rng = np.random.default_rng(seed)
    v = np.zeros((nd, nd, nd, nd, nqp), complex)
    base = rng.uniform(0.5, 1.0, (nd, nd))
    base = 0.5 * (base + base.T)
    for q in range(nqp):
        f = scale / (1.0 + q)
        for i in range(nd):
            for j in range(nd):
                v[i, j, i, j, q] = f * base[i, j]
    v += 0.01 * scale * (rng.standard_normal(v.shape) + 1j * rng.standard_normal(v.shape))
    return np.asfortranarray(v)


def test_oracle_read_vq_map():
    nd, nqp = 3, 4
    raw = seeded_vq(nd, nqp)
    v = O.read_vq_transform(raw)
    want = np.einsum("ijklq->ikljq", raw).reshape(nd * nd, nd * nd, nqp)
    assert rel_err(v, want) == 0.0


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_ladder_with_vq_matches_oracle(prec):
    p = problem("t3")
    s = p.spec
    raw = seeded_vq(s.ndim, s.nqp)
    inp = dataclasses.replace(to_inputs(p), vq=O.read_vq_transform(raw))
    nqw = s.nqp * (2 * s.iwb + 1)
    want = O.Oracle(inp).run(qw_points(p, 1, nqw))
    want.update(O.assemble(inp, want))
    with Ladder.from_problem(p) as lad:
        for iwb in range(-s.iwb, s.iwb + 1):
            lad.set_vertex(iwb, *p.vertex(iwb))
        lad.set_vq(raw)
        _, stats = lad.ladder_run(1, None, prec)
        out = lad.get_outputs()
        got = lad.assemble(out, p.siw)
    tol = 1e-10 if prec == "fp64" else 1e-8
    for k in ("chi_dens", "chi_magn", "sigma"):
        assert rel_err(got[k], want[k]) < tol, (k, rel_err(got[k], want[k]))
    assert rel_err(out["sigma_hf"], want["sigma_hf"]) < 1e-12
    assert np.abs(want["sigma_hf"]).max() > 0
    if prec == "mixed":
        assert stats["mixed_fallbacks"] == 0
