"""Derivatives of the ladder outputs (forward-mode tangents through the BSE,
the chi0 and EOM contractions; adga_ladder_run_tangent).

For each model parameter U, J (Kanamori, V = U - 2J) and the hopping scale t,
at fixed DMFT one-particle inputs:
  * the GPU tangent of chi_d/m(q, omega) and Sigma(k, nu) against central
    finite differences (h = 1e-5) of the GPU FP64 ladder, and
  * against central finite differences of the FP64 oracle (the dense
    reference: every output of the small grid);
both to 1e-6 relative (finite-difference truncation ~h^2, rounding ~1e-11).
"""
import dataclasses

import numpy as np
import pytest

from adga_b200 import Ladder, synth
from oracle import adga_oracle as O
from tests.helpers import problem, qw_points, rel_err, to_inputs

pytestmark = pytest.mark.gpu
KEYS = ("chi_dens", "chi_magn", "sigma")
H = 1e-5


def gpu_forward(p):
    s = p.spec
    with Ladder.from_problem(p) as lad:
        for iwb in range(-s.iwb, s.iwb + 1):
            lad.set_vertex(iwb, *p.vertex(iwb))
        lad.ladder_run(1, None, "fp64")
        return lad.assemble(lad.get_outputs(), p.siw)


def oracle_forward(p):
    s = p.spec
    inp = to_inputs(p)
    out = O.Oracle(inp).run(qw_points(p, 1, s.nqp * (2 * s.iwb + 1)))
    out.update(O.assemble(inp, out))
    return out


def gpu_tangent(p, par):
    s = p.spec
    dhk, du, dut, dvertex = synth.tangent_inputs(p, par)
    with Ladder.from_problem(p) as lad:
        for iwb in range(-s.iwb, s.iwb + 1):
            lad.set_vertex(iwb, *p.vertex(iwb))
            if dvertex is not None:
                lad.set_vertex_tangent(iwb, *dvertex(iwb))
        lad.set_tangent(dhk, du, dut)
        lad.ladder_run_tangent()
        fwd = lad.assemble(lad.get_outputs(), p.siw)
        tan = lad.assemble_tangent(lad.get_tangent_outputs())
    return fwd, tan


def fd(run, p, par):
    kw = {"U": "dU", "J": "dJ", "t": "dt"}[par]
    plus = run(synth.perturbed_problem(p, **{kw: H}))
    minus = run(synth.perturbed_problem(p, **{kw: -H}))
    return {k: (plus[k] - minus[k]) / (2 * H) for k in KEYS}


@pytest.mark.parametrize("name", ["t2", "t3"])
@pytest.mark.parametrize("par", synth.PARAMS)
def test_tangent_matches_gpu_finite_differences(name, par):
    p = problem(name)
    fwd, tan = gpu_tangent(p, par)
    ref = gpu_forward(p)
    for k in KEYS:                                   # the tangent run also gives the forward outputs
        assert rel_err(fwd[k], ref[k]) < 1e-13, k
    want = fd(gpu_forward, p, par)
    for k in KEYS:
        assert rel_err(tan[k], want[k]) < 1e-6, (par, k, rel_err(tan[k], want[k]))


@pytest.mark.parametrize("par", synth.PARAMS)
def test_tangent_matches_oracle_finite_differences(par):
    p = problem("t2")
    _, tan = gpu_tangent(p, par)
    want = fd(oracle_forward, p, par)
    for k in KEYS:
        assert rel_err(tan[k], want[k]) < 1e-6, (par, k, rel_err(tan[k], want[k]))
