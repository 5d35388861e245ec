"""CPU tests of the host side: the C-ABI library loads and exports every
declared entry point; host-only routines match the oracle; inputs are
deterministic.  No GPU compute is launched here."""
import re
from pathlib import Path

import numpy as np

import adga_b200
from adga_b200 import _lib, synth
from oracle import adga_oracle as O

ROOT = Path(__file__).resolve().parent.parent


def header_functions():
    text = (ROOT / "include" / "adga.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(adga_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    decl = header_functions()
    assert decl, "no declarations parsed"
    for name in decl:
        assert hasattr(lib, name), f"{name} declared in include/adga.h but not exported"
    assert sorted(_lib.EXPORTS) == decl


def test_create_u_c_abi_matches_golden():
    g = np.load(ROOT / "tests" / "golden" / "umatrix_example.npz")
    Um, u, ut = adga_b200.create_u(3, 5.0, 3.5, 0.75)
    np.testing.assert_array_equal(Um, g["Umat"])
    _, uo, uto = O.create_u([(3, 0)], [5.0], [3.5], [0.75])
    np.testing.assert_array_equal(u, uo)
    np.testing.assert_array_equal(ut, uto)


def test_generate_q_vol_c_abi():
    for nk, nq in [((20, 20, 20), (10, 10, 10)), ((6, 4, 2), (3, 2, 1)), ((12, 12, 12), (6, 6, 6))]:
        np.testing.assert_array_equal(adga_b200.generate_q_vol(nk, nq), O.generate_q_vol(nk, nq))


def test_generate_q_vol_rejects_mismatch():
    try:
        adga_b200.generate_q_vol((10, 10, 10), (3, 3, 3))
    except adga_b200.AdgaError:
        return
    raise AssertionError("mismatched grids accepted")


def test_synthetic_inputs_are_deterministic():
    a = synth.make_problem("t3")
    b = synth.make_problem("t3")
    np.testing.assert_array_equal(a.hk, b.hk)
    np.testing.assert_array_equal(a.giw, b.giw)
    np.testing.assert_array_equal(a.vertex(1)[0], b.vertex(1)[0])
    assert a.mu == b.mu


def test_synthetic_shapes_follow_reference_layouts():
    p = synth.make_problem("t5")
    s = p.spec
    assert p.hk.shape == (s.ndim, s.ndim, s.nkp) and p.hk.flags.f_contiguous
    assert p.siw.shape == (2 * p.iwmax, s.ndim)
    d, m = p.vertex(0)
    assert d.shape == (s.maxdim, s.maxdim) and d.flags.f_contiguous
    # Hermitian H(k)
    np.testing.assert_allclose(p.hk, np.conj(np.transpose(p.hk, (1, 0, 2))))
