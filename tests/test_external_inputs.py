"""External three-leg vertex and external local susceptibility
(external_threelegs / external_chi_loc, src/main.F90:407-411,560-561;
read_threeleg / read_chi_loc, src/hdf5_module.f90:776-994).

CPU: the oracle transforms against independent einsum restatements of their
index permutations where no disconnected term applies.
GPU: the transforms through the C ABI against the oracle (gamma^w through
adga_get_gamma_w, chi_loc through the outputs), and full FP64 ladders with
the external inputs against the oracle run with the same inputs (1e-10).
"""
import dataclasses

import numpy as np
import pytest

from adga_b200 import Ladder
from oracle import adga_oracle as O
from tests.helpers import problem, qw_points, rel_err, to_inputs


def raw_threeleg(nd, n3, seed, scale=1e-3):
    rng = np.random.default_rng(seed)
    sh = (nd, nd, nd, nd, 2 * n3)
    return [np.asfortranarray(rng.standard_normal(sh) + 1j * rng.standard_normal(sh)) * scale for _ in range(2)]


def raw_chi_loc(nd, n2, seed):
    rng = np.random.default_rng(seed)
    sh = (nd, nd, nd, nd, 2 * n2 + 1)
    return [np.asfortranarray(rng.standard_normal(sh) + 1j * rng.standard_normal(sh)) * 0.1 for _ in range(2)]


# ---------------------------------------------------------------- CPU
def test_oracle_threeleg_permutation_without_correlated_legs():
    p = problem("t3")
    s = p.spec
    nd, n3 = s.ndim, s.iwf + 1
    g3d, g3m = raw_threeleg(nd, n3, 1)
    gd, gm = O.read_threeleg_transform(g3d, g3m, 0, [[0, nd]], p.giw, p.n_dmft, p.beta, s.iwf, p.iwmax)
    # gamma(i1 = i nd + j, i2 = w nd2 + k nd + l) = beta g3(k, l, j, i, n3 + w - iwf)
    sl = g3d[..., n3 - s.iwf:n3 + s.iwf]                     # (k, l, j, i, w)
    want = p.beta * np.einsum("klijw->ijwkl", sl.transpose(0, 1, 3, 2, 4)).reshape(nd * nd, -1)
    assert rel_err(gd, want) < 1e-15


def test_oracle_chi_loc_permutation_without_extension():
    p = problem("t3")
    s = p.spec
    nd, n2 = s.ndim, s.iwb + 2
    cd, _ = raw_chi_loc(nd, n2, 2)
    out = O.read_chi_loc_transform(cd, "magn", [[nd, 0]], p.giw, p.n_dmft, p.beta, s.iwb, p.iwmax)
    # chi(i1 = i nd + j, i2 = k nd + l, w) = raw(i, j, l, k, n2 + w)
    sl = cd[..., n2 - s.iwb:n2 + s.iwb + 1]
    want = np.einsum("ijlkw->ijklw", sl).reshape(nd * nd, nd * nd, -1)
    assert rel_err(out, want) < 1e-15


# ---------------------------------------------------------------- GPU
NDIMS = [[[3, 0]], [[2, 1]], [[1, 1], [1, 0]]]


@pytest.mark.gpu
@pytest.mark.parametrize("ndims", NDIMS)
def test_threeleg_transform_matches_oracle(ndims):
    p = problem("t3")
    s = p.spec
    n3 = s.iwf + 2
    with Ladder.from_problem(p) as lad:
        for iwb in range(-s.iwb, s.iwb + 1):
            lad.set_vertex(iwb, *p.vertex(iwb))
            g3d, g3m = raw_threeleg(s.ndim, n3, 10 + iwb)
            lad.set_threeleg(iwb, g3d, g3m, ndims=ndims)
            gd, gm = lad.get_gamma_w(iwb)
            wd, wm = O.read_threeleg_transform(g3d, g3m, iwb, ndims, p.giw, p.n_dmft, p.beta, s.iwf, p.iwmax)
            assert rel_err(gd, wd) < 1e-13, (iwb, rel_err(gd, wd))
            assert rel_err(gm, wm) < 1e-13, (iwb, rel_err(gm, wm))


@pytest.mark.gpu
def test_ladder_with_external_threeleg_and_chi_loc_matches_oracle():
    p = problem("t3")
    s = p.spec
    ndims = [[2, 1]]
    n3, n2 = s.iwf + 1, s.iwb + 1
    raw3 = {iwb: raw_threeleg(s.ndim, n3, 20 + iwb) for iwb in range(-s.iwb, s.iwb + 1)}
    rcd, rcm = raw_chi_loc(s.ndim, n2, 5)
    gam = {iwb: O.read_threeleg_transform(*raw3[iwb], iwb, ndims, p.giw, p.n_dmft, p.beta, s.iwf, p.iwmax)
           for iwb in raw3}
    ext = (O.read_chi_loc_transform(rcd, "dens", ndims, p.giw, p.n_dmft, p.beta, s.iwb, p.iwmax),
           O.read_chi_loc_transform(rcm, "magn", ndims, p.giw, p.n_dmft, p.beta, s.iwb, p.iwmax))
    inp = dataclasses.replace(to_inputs(p), threeleg=lambda iwb: gam[iwb], chi_loc_ext=ext)
    nqw = s.nqp * (2 * s.iwb + 1)
    want = O.Oracle(inp).run(qw_points(p, 1, nqw))
    want.update(O.assemble(inp, want))
    with Ladder.from_problem(p) as lad:
        for iwb in range(-s.iwb, s.iwb + 1):
            lad.set_vertex(iwb, *p.vertex(iwb))
            lad.set_threeleg(iwb, *raw3[iwb], ndims=ndims)
        lad.set_chi_loc_ext(rcd, rcm, ndims=ndims)
        lad.ladder_run(1, None, "fp64")
        out = lad.get_outputs()
        got = lad.assemble(out, p.siw)
    assert rel_err(out["chi_loc_dens"], ext[0]) < 1e-13
    assert rel_err(out["chi_loc_magn"], ext[1]) < 1e-13
    for k in ("chi_dens", "chi_magn", "sigma", "chi_loc_dens"):
        assert rel_err(got[k], want[k]) < 1e-10, (k, rel_err(got[k], want[k]))
    assert rel_err(out["sigma_dmft"], want["sigma_dmft"]) < 1e-10
