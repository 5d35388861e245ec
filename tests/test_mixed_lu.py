"""The FP32 factorisation of the mixed path: without row interchanges (the
default; the BSE matrices have growth factor ~1), with them
(ADGA_MIXED_PIVOT=1), its panel products L21 / U12 on the tensor cores (the
default) or as FP32 CUDA-core tiles (ADGA_TRI_TILE=1), the triangular solves
on the tensor cores (the default) or streaming (ADGA_TRSV_STREAM=1), and the FP64 re-solve
of points whose refinement does not converge (ADGA_MAX_REFINE=1 leaves every
point unconverged); the refinement's two stopping rules: the bounded next
correction (default) and a solved one (ADGA_REFINE_EXACT=1)."""
import pytest

from adga_b200 import Ladder
from tests.helpers import library_env, oracle_run, problem, rel_err

pytestmark = pytest.mark.gpu


def run_mixed(p, settings):
    s = p.spec
    with library_env(settings):
        lad = Ladder.from_problem(p)
    try:
        for iwb in range(-s.iwb, s.iwb + 1):
            lad.set_vertex(iwb, *p.vertex(iwb))
        status, stats = lad.ladder_run(1, None, "mixed")
        out = lad.get_outputs()
        out.update(lad.assemble(out, p.siw))
        return status, stats, out
    finally:
        lad.close()


@pytest.mark.parametrize("name", ["t3b", "t3m", "t2"])
@pytest.mark.parametrize("pivot", ["0", "1"])
def test_mixed_factorisation_matches_oracle(name, pivot):
    p = problem(name)
    status, stats, got = run_mixed(p, {"ADGA_MIXED_PIVOT": pivot})
    want = oracle_run(p)
    assert stats["mixed_fallbacks"] == 0 and not status.any()
    for k in ("chi_dens", "chi_magn", "sigma"):
        assert rel_err(got[k], want[k]) < 1e-8, (k, rel_err(got[k], want[k]))


@pytest.mark.parametrize("name", ["t3b", "t3m", "t2", "c3s"])
@pytest.mark.parametrize("tri", ["tensor", "tile"])
def test_panel_products_match_oracle(name, tri):
    """L21 = A21 U11^-1 and U12 = L11^-1 A12 of every unpivoted step on the
    tensor cores (k_tc_tri, writing the update operands itself) or as FP32
    CUDA-core tiles with separate operand-split kernels: the same converged
    outputs, N = 144 .. 320 (partial last steps included)."""
    p = problem(name)
    status, stats, got = run_mixed(p, {"ADGA_TRI_TILE": "1"} if tri == "tile" else {})
    want = oracle_run(p)
    assert stats["mixed_fallbacks"] == 0 and not status.any()
    assert stats["max_refine_iters"] <= 3
    for k in ("chi_dens", "chi_magn", "sigma", "chi_qw_magn"):
        assert rel_err(got[k], want[k]) < 1e-8, (k, rel_err(got[k], want[k]))


@pytest.mark.parametrize("name", ["t2", "t3b", "t3m", "c3s"])
@pytest.mark.parametrize("solve", ["tensor", "stream"])
def test_triangular_solves_match_oracle(name, solve):
    """The solves with the FP32 factors (the back substitution after the LU, a
    forward and a back one per refinement sweep) on the tensor cores
    (k_trsv_tc, the default) or as streaming CUDA-core solves
    (ADGA_TRSV_STREAM=1): N = 24 .. 320, one to five row blocks, partial last
    blocks included; the refinement converges as fast as with FP32 solves."""
    p = problem(name)
    status, stats, got = run_mixed(p, {"ADGA_TRSV_STREAM": "1"} if solve == "stream" else {})
    want = oracle_run(p)
    assert stats["mixed_fallbacks"] == 0 and not status.any()
    assert stats["max_refine_iters"] <= 3 and stats["max_refine_resid"] <= 1e-10
    for k in ("chi_dens", "chi_magn", "sigma", "chi_qw_dens", "chi_qw_magn"):
        assert rel_err(got[k], want[k]) < 1e-8, (k, rel_err(got[k], want[k]))


@pytest.mark.parametrize("name", ["t3b", "t3m", "t2", "c3s", "t5"])
@pytest.mark.parametrize("resid", ["int8", "fp64"])
def test_refinement_residual_matches_oracle(name, resid):
    """The FP64 refinement residual r = B - X + (X D) F~ with its product formed
    exactly from int8 slices on the tensor cores (the default) or by the FP64
    CUDA-core GEMM (ADGA_RESID_FP64=1): the refinement converges without FP64
    re-solves to the same outputs."""
    p = problem(name)
    status, stats, got = run_mixed(p, {"ADGA_RESID_FP64": "1"} if resid == "fp64" else {})
    want = oracle_run(p)
    assert stats["mixed_fallbacks"] == 0 and not status.any()
    assert stats["max_refine_iters"] <= 3 and stats["max_refine_resid"] <= 1e-10
    for k in ("chi_dens", "chi_magn", "sigma", "chi_qw_dens", "chi_qw_magn"):
        assert rel_err(got[k], want[k]) < 1e-8, (k, rel_err(got[k], want[k]))


@pytest.mark.parametrize("pairs", [2, 3])
@pytest.mark.parametrize("name", ["t3b", "t3m", "c3s"])
def test_delayed_groups_match_oracle(name, pairs):
    """tune pairs = 2 / 3: the tensor-core updates delayed in groups of three /
    four steps (the next step's strips after each step, the rest with a K = G * 6
    NB product from G operand stagings).  Groups of three: N = 144 (one group
    ending at the last step), 216 (a group and a lone step), 320 (a group and a
    pair); groups of four: 144 (a partial group), 216 (one group ending at the
    last step), 320 (a group and a lone step)."""
    p = problem(name)
    s = p.spec
    with library_env({}):
        lad = Ladder.from_problem(p)
    try:
        for iwb in range(-s.iwb, s.iwb + 1):
            lad.set_vertex(iwb, *p.vertex(iwb))
        lad.tune = {"pairs": pairs}
        status, stats = lad.ladder_run(1, None, "mixed")
        got = lad.get_outputs()
        got.update(lad.assemble(got, p.siw))
    finally:
        lad.close()
    want = oracle_run(p)
    assert stats["mixed_fallbacks"] == 0 and not status.any()
    assert stats["max_refine_iters"] <= 3
    for k in ("chi_dens", "chi_magn", "sigma", "chi_qw_dens", "chi_qw_magn"):
        assert rel_err(got[k], want[k]) < 1e-8, (k, rel_err(got[k], want[k]))


@pytest.mark.parametrize("name", ["t3b", "t3m"])
def test_step_by_step_updates_match_oracle(name):
    """ADGA_NO_PAIRS=1: the unpivoted FP32 factorisation with one tensor-core
    update per step instead of the delayed pair updates."""
    p = problem(name)
    status, stats, got = run_mixed(p, {"ADGA_NO_PAIRS": "1"})
    want = oracle_run(p)
    assert stats["mixed_fallbacks"] == 0 and not status.any()
    for k in ("chi_dens", "chi_magn", "sigma"):
        assert rel_err(got[k], want[k]) < 1e-8, (k, rel_err(got[k], want[k]))


def test_unconverged_points_are_resolved_in_fp64():
    p = problem("t3m")
    status, stats, got = run_mixed(p, {"ADGA_MAX_REFINE": "1"})
    npts = p.spec.nqp * (2 * p.spec.iwb + 1)
    assert stats["mixed_fallbacks"] == npts
    assert (status == -1).all()
    want = oracle_run(p)
    for k in ("chi_dens", "chi_magn", "sigma"):
        assert rel_err(got[k], want[k]) < 1e-10, (k, rel_err(got[k], want[k]))


@pytest.mark.parametrize("exact", ["0", "1"])
def test_refinement_stopping_rules(exact):
    p = problem("t3m")
    status, stats, got = run_mixed(p, {"ADGA_REFINE_EXACT": exact})
    want = oracle_run(p)
    assert stats["mixed_fallbacks"] == 0 and not status.any()
    assert stats["max_refine_resid"] <= 1e-10
    for k in ("chi_dens", "chi_magn", "sigma"):
        assert rel_err(got[k], want[k]) < (1e-12 if exact == "1" else 1e-9), (k, rel_err(got[k], want[k]))
