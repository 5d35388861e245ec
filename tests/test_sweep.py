"""The uneven-size parameter sweep (adga_b200.sweep) on shrunken parameter
points: mixed ladder + gradients in U and J per point, the FP64 check pass,
and one point against the oracle."""
import dataclasses

import pytest

from adga_b200 import sweep, synth
from oracle import adga_oracle as O
from tests.helpers import qw_points, rel_err, to_inputs

pytestmark = pytest.mark.gpu


def small_specs():
    """The first sweep points (ndim 1, 3, 5 mixed) on a 4^3 k / 2^3 q grid, 2 x 6 fermionic, 3 bosonic."""
    return [dataclasses.replace(sp, nk=(4, 4, 4), nq=(2, 2, 2), iwf=min(sp.iwf, 6), iwb=1)
            for sp in synth.sweep_specs(6)]


def test_sweep_runs_uneven_points_with_gradients():
    specs = small_specs()
    assert len({sp.ndim for sp in specs}) > 1
    res = sweep.run_sweep(specs)
    s = res["summary"]
    assert s["parameter_points"] == len(specs)
    assert s["qw_points"] == sum(sp.nqp * (2 * sp.iwb + 1) for sp in specs)
    Ns = [r["N"] for r in res["points"]]
    assert Ns == sorted(Ns, reverse=True)                 # largest BSE dimension first
    # kernel choices tuned once per (orbital count, BSE size), every point runs with its size's choice
    assert set(s["tune"]) == {f"ndim{r['ndim']}_N{r['N']}" for r in res["points"]}
    for r in res["points"]:
        assert r["tune"] == s["tune"][f"ndim{r['ndim']}_N{r['N']}"]
    for r in res["points"]:
        assert r["mixed_fallbacks"] == 0
        for k, e in r["err_vs_fp64"].items():
            assert e < 1e-9, (r["name"], k, e)


def test_sweep_point_matches_oracle():
    sp = [s for s in small_specs() if s.ndim == 3][0]
    prepared = sweep._prepare(sp, [-1, 0, 1])
    rec = sweep.run_point(prepared, [-1, 0, 1], check_fp64=False, keep=True)
    prob = prepared[0]
    s = prob.spec
    inp = to_inputs(prob)
    want = O.Oracle(inp).run(qw_points(prob, 1, s.nqp * (2 * s.iwb + 1)))
    want.update(O.assemble(inp, want))
    for k in ("chi_dens", "chi_magn", "sigma"):
        assert rel_err(rec["mixed"][k], want[k]) < 1e-8, (k, rel_err(rec["mixed"][k], want[k]))
