"""get_outputs into caller-owned (pinned) host arrays gives the same
accumulators as freshly allocated ones, and rejects mismatched arrays."""
import numpy as np
import pytest
import torch

from adga_b200 import Ladder
from tests.helpers import problem

pytestmark = pytest.mark.gpu


def test_get_outputs_into_pinned_arrays():
    p = problem("t3")
    s = p.spec
    with Ladder.from_problem(p) as lad:
        for iwb in range(-s.iwb, s.iwb + 1):
            lad.set_vertex(iwb, *p.vertex(iwb))
        lad.ladder_run(1, None, "fp64")
        want = lad.get_outputs()
        out = {k: torch.empty(int(np.prod(sh)), dtype=torch.complex128).pin_memory().numpy().reshape(sh, order="F")
               for k, sh in lad.output_shapes().items()}
        got = lad.get_outputs(out=out)
        assert got is out
        for k in want:
            np.testing.assert_array_equal(got[k], want[k])
        bad = dict(out, sigma_nl=np.zeros(out["sigma_nl"].shape, dtype=np.complex128))   # C order
        with pytest.raises(ValueError):
            lad.get_outputs(out=bad)
