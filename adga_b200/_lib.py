"""ctypes binding of libadga_b200.so (the C ABI declared in include/adga.h).

The library is loaded from the package directory only; there is no fallback:
if it is missing, every call raises.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libadga_b200.so"

ADGA_FP64, ADGA_MIXED = 0, 1
ADGA_ENOCONV = -6
ERRORS = {-1: "ADGA_EINVAL", -2: "ADGA_ECUDA", -3: "ADGA_ENOMEM", -4: "ADGA_ETIMEOUT",
          -5: "ADGA_ESTATE", -6: "ADGA_ENOCONV"}

# exported entry points (kept in sync with include/adga.h)
EXPORTS = [
    "adga_create", "adga_destroy", "adga_last_error", "adga_device_bytes", "adga_set_vertex",
    "adga_reset_outputs", "adga_ladder_run", "adga_get_outputs", "adga_get_chi0_loc",
    "adga_get_chi0_loc_inv", "adga_chi0_q", "adga_bse_point", "adga_get_gamma_w",
    "adga_calc_chi_qw", "adga_calc_eom_dynamic", "adga_calc_eom_dmft", "adga_calc_eom_static",
    "adga_inverse_matrix_z", "adga_index_kq", "adga_generate_q_vol", "adga_create_u",
    "adga_inverse_matrix_z_noalloc", "adga_set_vertex_g4", "adga_vertex_transform",
    "adga_index2component_band", "adga_post_loop", "adga_set_threeleg", "adga_set_chi_loc_ext",
    "adga_set_vq", "adga_set_tangent", "adga_set_vertex_tangent", "adga_ladder_run_tangent",
    "adga_get_tangent_outputs", "adga_clear_tangents", "adga_set_tune", "adga_get_tune",
    "adga_autotune",
]


class Dims(C.Structure):
    _fields_ = [("ndim", C.c_int), ("nkpx", C.c_int), ("nkpy", C.c_int), ("nkpz", C.c_int),
                ("nqpx", C.c_int), ("nqpy", C.c_int), ("nqpz", C.c_int), ("iwmax", C.c_int),
                ("iwfmax_small", C.c_int), ("iwbmax_small", C.c_int), ("iwstart", C.c_int),
                ("iwstop", C.c_int), ("do_chi", C.c_int), ("do_eom", C.c_int),
                ("nkp_eom", C.c_int), ("beta", C.c_double), ("mu", C.c_double)]


class RunStats(C.Structure):
    _fields_ = [("points", C.c_int), ("lu_info_nonzero", C.c_int), ("mixed_fallbacks", C.c_int),
                ("max_refine_iters", C.c_int), ("max_refine_resid", C.c_double),
                ("ms_total", C.c_double), ("ms_chi0", C.c_double), ("ms_bse", C.c_double),
                ("ms_lu", C.c_double), ("ms_post", C.c_double), ("ms_eom", C.c_double),
                ("kernel_launches", C.c_longlong), ("ms_trail", C.c_double),
                ("trail_gflop", C.c_double), ("trail_launches", C.c_int),
                ("trail_gbytes", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Tune(C.Structure):
    _fields_ = [("factor", C.c_int), ("pairs", C.c_int), ("tri_tc", C.c_int), ("batch", C.c_int),
                ("resid", C.c_int), ("trsv_tc", C.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class TuneTrial(C.Structure):
    _fields_ = [("tune", Tune), ("ms", C.c_double), ("err", C.c_double), ("accepted", C.c_int)]


class Outputs(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in ("chi_qw_dens", "chi_qw_magn", "bubble_nl", "bubble_loc",
                                          "chi_loc_dens", "chi_loc_magn", "sigma_nl",
                                          "sigma_dmft", "sigma_hf")]


_lib = None


def load():
    """Load the library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH} is missing: run `python -m adga_b200.build` "
                           "(there is no CPU fallback for the ladder hot path)")
    lib = C.CDLL(str(LIB_PATH))
    vp, ip, i, d = C.c_void_p, C.POINTER(C.c_int), C.c_int, C.c_double
    sig = {
        "adga_create": [C.POINTER(Dims), vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, C.POINTER(vp)],
        "adga_destroy": [vp],
        "adga_device_bytes": [vp, C.POINTER(C.c_longlong)],
        "adga_set_vertex": [vp, i, vp, vp],
        "adga_reset_outputs": [vp],
        "adga_ladder_run": [vp, i, i, i, ip, C.POINTER(RunStats)],
        "adga_get_outputs": [vp, C.POINTER(Outputs)],
        "adga_get_chi0_loc": [vp, i, i, vp],
        "adga_get_chi0_loc_inv": [vp, i, i, vp],
        "adga_chi0_q": [vp, i, i, vp, vp],
        "adga_bse_point": [vp, i, i, i, vp, vp, vp, ip],
        "adga_get_gamma_w": [vp, i, vp, vp],
        "adga_calc_chi_qw": [vp, vp, vp, vp],
        "adga_calc_eom_dynamic": [vp, vp, vp, vp, i, i, vp],
        "adga_calc_eom_dmft": [vp, vp, i, vp],
        "adga_calc_eom_static": [vp, i, vp],
        "adga_inverse_matrix_z": [vp, i, ip, C.c_char_p],
        "adga_inverse_matrix_z_noalloc": [vp, vp, i, ip, vp],
        "adga_index_kq": [i, i, i, vp, i, vp, i, vp],
        "adga_generate_q_vol": [i, i, i, i, i, i, vp],
        "adga_create_u": [i, d, d, d, vp, vp, vp],
        "adga_set_vertex_g4": [vp, i, i, i, i, vp, vp, vp],
        "adga_vertex_transform": [vp, i, i, i, i, vp, vp, vp, vp, vp],
        "adga_index2component_band": [i, i, vp],
        "adga_post_loop": [vp, vp, vp, vp, vp, vp],
        "adga_set_threeleg": [vp, i, i, i, vp, vp, vp],
        "adga_set_chi_loc_ext": [vp, i, i, vp, vp, vp],
        "adga_set_vq": [vp, vp],
        "adga_set_tangent": [vp, i, vp, vp, vp],
        "adga_set_vertex_tangent": [vp, i, i, vp, vp],
        "adga_ladder_run_tangent": [vp, i, i, i, ip, C.POINTER(RunStats)],
        "adga_get_tangent_outputs": [vp, i, C.POINTER(Outputs)],
        "adga_clear_tangents": [vp],
        "adga_set_tune": [vp, C.POINTER(Tune)],
        "adga_get_tune": [vp, C.POINTER(Tune)],
        "adga_autotune": [vp, i, i, d, C.POINTER(TuneTrial), i, ip, C.POINTER(Tune)],
    }
    for name, args in sig.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = C.c_int
    lib.adga_last_error.argtypes = [vp]
    lib.adga_last_error.restype = C.c_char_p
    _lib = lib
    return lib


def ptr(a):
    return None if a is None else C.c_void_p(a.ctypes.data)
