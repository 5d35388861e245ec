"""Vertex ingest: read_vertex's compound-index transform (src/hdf5_module.f90:629-773).

CPU: the oracle restatement against known answers (zero connected vertex ->
the local bubble; a round trip chi_loc -> g4 -> chi_loc) and the C-ABI group
decode against index2component_band (src/aux.f90:169-186).
GPU: adga_vertex_transform against the oracle for every vertex type, for one
and two inequivalent atoms with uncorrelated bands, at omega = 0 and != 0;
a full ladder fed through adga_set_vertex_g4 against the same ladder fed
through adga_set_vertex, and against the oracle (FP64 tolerance 1e-10).
"""
import numpy as np
import pytest

from adga_b200 import Ladder, ladder as L
from oracle import adga_oracle as O
from tests.helpers import oracle_run, problem, rel_err

TYPES = [O.FULL_G4, O.CONNECTED_G4, O.CHI_G4]


def random_g4(nd, W, seed):
    rng = np.random.default_rng(seed)
    shape = (nd, nd, 2 * W, nd, nd, 2 * W)
    return [np.asfortranarray(rng.standard_normal(shape) + 1j * rng.standard_normal(shape)) * 1e-3
            for _ in range(2)]


def chi_to_connected_g4(chi, iwb, giw, beta, iwf, iwmax, nd, W):
    """Inverse of the connected-G4 transform: g4 such that read_vertex returns chi."""
    nd2 = nd * nd
    g4 = np.zeros((nd, nd, 2 * W, nd, nd, 2 * W), complex, order="F")
    for i2 in range(chi.shape[1]):
        w2, r2 = divmod(i2, nd2)
        l, k = divmod(r2, nd)
        for i1 in range(chi.shape[0]):
            w1, r1 = divmod(i1, nd2)
            i, j = divmod(r1, nd)
            v = chi[i1, i2]
            if w1 == w2 and i == l and j == k:
                v = v + beta * giw[w1 - iwf + iwmax, i] * giw[w2 - iwf - iwb + iwmax, j]
            g4[i, j, w1 - iwf + W, k, l, w2 - iwf + W] = v / beta
    return g4


# ---------------------------------------------------------------- CPU
def test_oracle_zero_connected_vertex_is_local_bubble():
    p = problem("t3")
    s = p.spec
    nd, W = s.ndim, s.iwf + 1
    z = np.zeros((nd, nd, 2 * W, nd, nd, 2 * W), complex)
    for iwb in (0, 1):
        cd, cm = O.read_vertex_transform(z, z, iwb, O.CONNECTED_G4, [[nd, 0]], p.giw, p.beta, s.iwf, p.iwmax)
        nd2 = nd * nd
        want = np.zeros(cd.shape[0], complex)
        for i1 in range(cd.shape[0]):
            w, r = divmod(i1, nd2)
            i, j = divmod(r, nd)
            want[i1] = -p.beta * p.giw[w - s.iwf + p.iwmax, i] * p.giw[w - s.iwf - iwb + p.iwmax, j]
        assert np.array_equal(cd, cm)
        assert np.allclose(cd, np.diag(want), rtol=0, atol=1e-15 * np.abs(want).max())


def test_oracle_connected_round_trip():
    p = problem("t3")
    s = p.spec
    nd, W = s.ndim, s.iwf + 2
    chi_d, chi_m = p.vertex(1)
    g4d = chi_to_connected_g4(chi_d, 1, p.giw, p.beta, s.iwf, p.iwmax, nd, W)
    g4m = chi_to_connected_g4(chi_m, 1, p.giw, p.beta, s.iwf, p.iwmax, nd, W)
    cd, cm = O.read_vertex_transform(g4d, g4m, 1, O.CONNECTED_G4, [[nd, 0]], p.giw, p.beta, s.iwf, p.iwmax)
    assert rel_err(cd, chi_d) < 1e-14 and rel_err(cm, chi_m) < 1e-14


def test_index2component_band_c_abi():
    for nb in (1, 2, 3, 5):
        for ind in range(1, nb ** 4 + 1):
            b = L.index2component_band(nb, ind)
            assert b == O.index2component_band(nb, ind)
            assert O.component2index_band(nb, *b) == ind
    with pytest.raises(L.AdgaError):
        L.index2component_band(3, 82)


# ---------------------------------------------------------------- GPU
@pytest.mark.gpu
@pytest.mark.parametrize("ndims", [[[3, 0]], [[2, 1]], [[1, 1], [1, 0]]])
@pytest.mark.parametrize("iwb", [0, 1, -1])
def test_vertex_transform_matches_oracle(ndims, iwb):
    p = problem("t3")
    s = p.spec
    W = s.iwf + 2
    g4d, g4m = random_g4(s.ndim, W, seed=7 + iwb)
    with Ladder.from_problem(p) as lad:
        for vt in TYPES:
            gd, gm = lad.vertex_transform(iwb, g4d, g4m, vertex_type=vt, ndims=ndims)
            wd, wm = O.read_vertex_transform(g4d, g4m, iwb, vt, ndims, p.giw, p.beta, s.iwf, p.iwmax)
            assert rel_err(gd, wd) < 1e-14, (vt, rel_err(gd, wd))
            assert rel_err(gm, wm) < 1e-14, (vt, rel_err(gm, wm))


@pytest.mark.gpu
def test_vertex_transform_rejects_bad_arguments():
    p = problem("t3")
    s = p.spec
    with Ladder.from_problem(p) as lad:
        g4d, g4m = random_g4(s.ndim, s.iwf - 1, seed=1)        # box smaller than the small box
        with pytest.raises(L.AdgaError):
            lad.vertex_transform(0, g4d, g4m)
        g4d, g4m = random_g4(s.ndim, s.iwf, seed=1)
        with pytest.raises(L.AdgaError):
            lad.vertex_transform(0, g4d, g4m, vertex_type=3)
        with pytest.raises(L.AdgaError):
            lad.vertex_transform(0, g4d, g4m, ndims=[[2, 0]])   # bands do not add up to ndim


@pytest.mark.gpu
def test_ladder_through_vertex_ingest_matches_set_vertex_and_oracle():
    p = problem("t3")
    s = p.spec
    W = s.iwf + 1
    ref = oracle_run(p)
    outs = []
    for use_g4 in (False, True):
        with Ladder.from_problem(p) as lad:
            for iwb in range(-s.iwb, s.iwb + 1):
                chi_d, chi_m = p.vertex(iwb)
                if use_g4:
                    g4d = chi_to_connected_g4(chi_d, iwb, p.giw, p.beta, s.iwf, p.iwmax, s.ndim, W)
                    g4m = chi_to_connected_g4(chi_m, iwb, p.giw, p.beta, s.iwf, p.iwmax, s.ndim, W)
                    lad.set_vertex_g4(iwb, g4d, g4m, vertex_type="connected_g4")
                else:
                    lad.set_vertex(iwb, chi_d, chi_m)
            lad.ladder_run(1, None, "fp64")
            out = lad.get_outputs()
            outs.append(lad.assemble(out, p.siw))
    for k in ("chi_dens", "chi_magn", "sigma"):
        assert rel_err(outs[1][k], outs[0][k]) < 1e-13, k
        assert rel_err(outs[1][k], ref[k]) < 1e-10, k
