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


class _FakeSpec:
    name, ndim, iwf, beta, U, J, nqp, iwb = "fake", 1, 2, 10.0, 2.0, 0.0, 3, 1


class _FakeProblem:
    spec = _FakeSpec()
    siw = None


class _FakeLadder:
    """Stands in for the library: the mixed pass of a point fails with the given
    error code (the tangent refinement's non-convergence is ADGA_ENOCONV); the
    FP64 pass returns fixed outputs.  Records the precisions it was run with."""
    fail_code = sweep.ADGA_ENOCONV
    runs = []

    @classmethod
    def from_problem(cls, prob):
        return cls()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return False

    tune = {"factor": 0}

    def set_vertex(self, *a): pass
    def set_tangent(self, *a, **k): pass
    def set_vertex_tangent(self, *a, **k): pass
    def reset_outputs(self): pass

    def ladder_run_tangent(self, qs, qe, precision):
        _FakeLadder.runs.append(precision)
        if precision == "mixed":
            raise sweep.AdgaError(self.fail_code, "tangent refinement did not converge")
        return None, {"ms_total": 2.0, "max_refine_iters": 0, "mixed_fallbacks": 0}

    def get_outputs(self):
        return {"chi_qw_dens": np.zeros((1, 1, 3)), "chi_qw_magn": np.zeros((1, 1, 3))}

    def assemble(self, raw, siw):
        return {"chi_dens": np.ones(3), "chi_magn": np.ones(3), "sigma": np.ones(2)}

    def get_tangent_outputs(self, d):
        return {}

    def assemble_tangent(self, raw):
        return {"chi_magn": np.ones(3), "sigma": np.ones(2)}


def test_point_reruns_in_fp64_when_tangents_do_not_converge(monkeypatch):
    monkeypatch.setattr(sweep, "Ladder", _FakeLadder)
    _FakeLadder.runs = []
    _FakeLadder.fail_code = sweep.ADGA_ENOCONV
    prepared = (_FakeProblem(), {0: (None, None)}, [(None, None, None, None)] * len(sweep.GRAD_PARAMS))
    rec = sweep.run_point(prepared, [0], check_fp64=True)
    # the mixed pass failed, the point's pass ran again in FP64 (its time counts as the
    # point's mixed time), then the FP64 reference pass ran
    assert _FakeLadder.runs == ["mixed", "fp64", "fp64"]
    assert "did not converge" in rec["fp64_pass"]
    assert rec["ms_mixed"] == 2.0 and rec["points"] == 3
    assert rec["err_vs_fp64"]["chi_magn"] == 0.0


def test_point_passes_other_library_errors_on(monkeypatch):
    monkeypatch.setattr(sweep, "Ladder", _FakeLadder)
    _FakeLadder.runs = []
    _FakeLadder.fail_code = -1                      # ADGA_EINVAL: not a convergence failure
    prepared = (_FakeProblem(), {0: (None, None)}, [(None, None, None, None)] * len(sweep.GRAD_PARAMS))
    try:
        sweep.run_point(prepared, [0], check_fp64=False)
    except sweep.AdgaError as e:
        assert e.code == -1
    else:
        raise AssertionError("the library error was swallowed")
    assert _FakeLadder.runs == ["mixed"]
