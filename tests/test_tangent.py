"""Derivatives of the ladder outputs (forward-mode tangents through the BSE,
the chi0 and EOM contractions; adga_ladder_run_tangent), FP64 and mixed.

For each model parameter U, J (Kanamori, V = U - 2J) and the hopping scale t,
at fixed DMFT one-particle inputs:
  * the GPU tangent of chi_d/m(q, omega) and Sigma(k, nu) against central
    finite differences (h = 1e-5) of the GPU FP64 ladder, and
  * against central finite differences of the FP64 oracle (the dense
    reference: every output of the small grid);
both to 1e-6 relative (finite-difference truncation ~h^2, rounding ~1e-11).
"""
from functools import lru_cache

import numpy as np
import pytest

from adga_b200 import Ladder, synth
from oracle import adga_oracle as O
from tests.helpers import library_env, problem, qw_points, rel_err, to_inputs

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


def gpu_tangent(p, par, precision="fp64"):
    s = p.spec
    dhk, du, dut, dvertex = synth.tangent_inputs(p, par)
    with Ladder.from_problem(p) as lad:
        for iwb in range(-s.iwb, s.iwb + 1):
            lad.set_vertex(iwb, *p.vertex(iwb))
            if dvertex is not None:
                lad.set_vertex_tangent(iwb, *dvertex(iwb))
        lad.set_tangent(dhk, du, dut)
        lad.ladder_run_tangent(precision=precision)
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


@pytest.mark.parametrize("name", ["t2", "t3m"])
@pytest.mark.parametrize("par", synth.PARAMS)
def test_mixed_tangent_matches_fp64(name, par):
    """FP32 factors with FP64 refinement of the tangent solves: the tangents (and
    the forward outputs of the same run) agree with the FP64 path to the
    refinement's tolerance."""
    p = problem(name)
    f64, t64 = gpu_tangent(p, par, "fp64")
    fmx, tmx = gpu_tangent(p, par, "mixed")
    for k in KEYS:
        assert rel_err(fmx[k], f64[k]) < 1e-9, (k, rel_err(fmx[k], f64[k]))
        assert rel_err(tmx[k], t64[k]) < 1e-9, (par, k, rel_err(tmx[k], t64[k]))


def c3s_pick(out, s):
    w0 = s.iwb * s.nqp + np.arange(s.nqp)
    return out["chi_magn"][:, :, w0], out["sigma"]


@lru_cache(maxsize=None)
def c3s_oracle_jacobian():
    """Central differences (h = 1e-5, the 4-point stencil
    (-f(2h) + 8 f(h) - 8 f(-h) + f(-2h)) / 12h) of the oracle's chi_m(q, omega=0)
    and Sigma on the differentiation model's 4^3 sub-grid, one column per
    parameter.  chi_m is large and steep in U at beta = 20, where the 2-point
    quotient's h^2 truncation alone reaches 1e-5 relative."""
    p = problem("c3s")
    cols = {}
    for par, kw in zip(synth.PARAMS, ("dU", "dJ", "dt")):
        f = {m: c3s_pick(oracle_forward(synth.perturbed_problem(p, **{kw: m * H})), p.spec) for m in (-2, -1, 1, 2)}
        cols[par] = tuple((-f[2][i] + 8 * f[1][i] - 8 * f[-1][i] + f[-2][i]) / (12 * H) for i in range(2))
    return cols


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_c3_subgrid_tangents_match_oracle_dense_jacobian(precision):
    """dchi_m(q, omega=0)/dU, /dJ and dSigma/dU, /dt (every parameter, both outputs) on
    the differentiation model (2 e_g orbitals, beta = 20, 2 x 40 fermionic and 11
    bosonic frequencies, BSE 320 x 320) restricted to a 4^3 k / 2^3 q grid."""
    p = problem("c3s")
    jac = c3s_oracle_jacobian()
    for par in synth.PARAMS:
        _, tan = gpu_tangent(p, par, precision)
        dchi, dsig = c3s_pick(tan, p.spec)
        wchi, wsig = jac[par]
        assert rel_err(dchi, wchi) < 1e-6, (par, "chi_m", rel_err(dchi, wchi))
        assert rel_err(dsig, wsig) < 1e-6, (par, "sigma", rel_err(dsig, wsig))


def test_mixed_tangents_of_points_resolved_in_fp64():
    """ADGA_MAX_REFINE=1 leaves every mixed point unconverged: each is re-solved
    in FP64 together with its tangents, which then equal the FP64 path's."""
    p = problem("t3m")
    _, t64 = gpu_tangent(p, "U", "fp64")
    with library_env({"ADGA_MAX_REFINE": "1"}):
        _, tmx = gpu_tangent(p, "U", "mixed")
    for k in KEYS:
        assert rel_err(tmx[k], t64[k]) < 1e-12, (k, rel_err(tmx[k], t64[k]))
