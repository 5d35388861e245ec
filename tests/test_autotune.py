"""The mixed path's kernel choices (adga_set_tune / adga_get_tune) and the
autotuner that picks them by measurement (adga_autotune): every candidate is
timed on a sample of the handle's own points and checked against the FP64
path; the fastest one within the tolerance is kept on the handle."""
import numpy as np
import pytest

from adga_b200 import Ladder
from adga_b200.ladder import AdgaError
from tests.helpers import library_env, oracle_run, problem, rel_err

pytestmark = pytest.mark.gpu


def make_ladder(p):
    s = p.spec
    with library_env({}):
        lad = Ladder.from_problem(p)
    for iwb in range(-s.iwb, s.iwb + 1):
        lad.set_vertex(iwb, *p.vertex(iwb))
    return lad


def test_tune_round_trip_and_validation():
    lad = make_ladder(problem("t3"))
    try:
        assert lad.tune == {"factor": 0, "pairs": 2, "tri_tc": 1, "batch": 0, "resid": 1, "trsv_tc": 1}
        lad.tune = {"pairs": 0, "batch": 3}
        assert lad.tune == {"factor": 0, "pairs": 0, "tri_tc": 1, "batch": 3, "resid": 1, "trsv_tc": 1}
        for bad in ({"factor": 2}, {"pairs": -1}, {"pairs": 4}, {"batch": -5}, {"resid": 2}, {"trsv_tc": 3}):
            with pytest.raises(AdgaError):
                lad.tune = bad
        assert lad.tune["batch"] == 3
    finally:
        lad.close()


@pytest.mark.parametrize("name", ["t3m", "c3s"])
def test_autotune_picks_the_fastest_accurate_configuration(name):
    p = problem(name)
    s = p.spec
    lad = make_ladder(p)
    try:
        q0 = s.iwb * s.nqp + 1                      # the omega = 0 slice as the sample
        best, trials = lad.autotune(q0, q0 + s.nqp - 1)
        # the tensor-core variants (panel products, groups of two, three or four, int8 or FP64
        # residual, tensor-core or streaming solves) + the FP64 factorisation
        assert len(trials) == 8
        assert all(t["accepted"] and t["err"] <= 1e-8 for t in trials), trials
        fastest = min(trials, key=lambda t: t["ms"])
        assert best == {k: fastest[k] for k in ("factor", "pairs", "tri_tc", "batch", "resid", "trsv_tc")}
        assert lad.tune == best
        # the accumulators were reset; the tuned mixed run still matches the oracle
        status, stats = lad.ladder_run(1, None, "mixed")
        out = lad.get_outputs()
        out.update(lad.assemble(out, p.siw))
        want = oracle_run(p)
        for k in ("chi_dens", "chi_magn", "sigma"):
            assert rel_err(out[k], want[k]) < 1e-8, (k, rel_err(out[k], want[k]))
    finally:
        lad.close()


def test_fp64_factorisation_choice_equals_the_fp64_path():
    p = problem("t3m")
    lad = make_ladder(p)
    try:
        lad.ladder_run(1, None, "fp64")
        ref = lad.get_outputs()
        lad.reset_outputs()
        lad.tune = {"factor": 1}
        status, stats = lad.ladder_run(1, None, "mixed")
        got = lad.get_outputs()
        assert stats["mixed_fallbacks"] == 0 and stats["max_refine_iters"] == 0
        for k in ("chi_qw_dens", "chi_qw_magn", "sigma_nl"):
            np.testing.assert_array_equal(got[k], ref[k])
    finally:
        lad.close()


def test_batch_choice_splits_the_run():
    """batch = 3 on an 8-point slice: three batches, the same outputs."""
    p = problem("t3m")
    lad = make_ladder(p)
    try:
        lad.ladder_run(1, None, "mixed")
        ref = lad.get_outputs()
        lad.reset_outputs()
        lad.tune = {"batch": 3}
        lad.ladder_run(1, None, "mixed")
        got = lad.get_outputs()
        for k in ("chi_qw_dens", "chi_qw_magn", "sigma_nl"):
            assert rel_err(got[k], ref[k]) < 1e-9, k
    finally:
        lad.close()
