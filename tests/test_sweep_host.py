"""Host logic of the parameter sweep (no GPU): the seeded parameter draws of
the sweep configuration, the compound (q, omega) ranges of the omega slices,
and the differentiation model's sub-grid problem."""
import numpy as np

from adga_b200 import sweep, synth


def test_sweep_specs_follow_the_configuration():
    specs = synth.sweep_specs(64)
    assert len(specs) == 64
    assert {sp.ndim for sp in specs} <= {1, 3, 5} and len({sp.ndim for sp in specs}) == 3
    for sp in specs:
        assert 2.0 <= sp.U <= 6.0
        if sp.ndim > 1:
            assert 0.1 <= sp.J / sp.U <= 0.2
        assert sp.beta in (10.0, 20.0, 40.0) and sp.iwf in (20, 40, 80)
        assert sp.nk == (12, 12, 12) and sp.nq == (6, 6, 6) and 2 * sp.iwb + 1 == 11
    Ns = {sp.ndim ** 2 * 2 * sp.iwf for sp in specs}
    assert min(Ns) == 40 and max(Ns) == 4000
    again = synth.sweep_specs(64)                   # seeded
    assert [(s.ndim, s.U, s.J, s.beta, s.iwf) for s in again] == [(s.ndim, s.U, s.J, s.beta, s.iwf) for s in specs]


def test_compound_ranges_of_omega_slices():
    # 1-based compound index qw = (iwb + iwbmax) * nqp + iq, omega outer
    assert sweep._ranges(8, 2, [0]) == [(17, 24)]
    assert sweep._ranges(8, 2, [1, -2]) == [(1, 8), (25, 32)]
    r = sweep._ranges(216, 5, range(-5, 6))
    assert r[0] == (1, 216) and r[-1] == (10 * 216 + 1, 11 * 216)


def test_differentiation_subgrid_problem():
    p = synth.make_problem("c3s")
    s = p.spec
    assert s.ndim == 2 and s.nk == (4, 4, 4) and s.nq == (2, 2, 2) and s.iwf == 40 and s.beta == 20.0
    d, m = p.vertex(0)
    assert d.shape == (320, 320) and np.isfinite(d).all() and np.isfinite(m).all()
    dhk, du, dut, dvertex = synth.tangent_inputs(p, "U")
    assert dhk is None and dvertex is not None and du.shape == (4, 4)
