"""Host-side mirror of the reference's hot-path routines over the C ABI.

The reference is Fortran called from its own main loop; this module gives the
same operations to Python callers with the reference's names, argument
meanings, array shapes (Fortran order, 0-based Python indices) and error
behaviour (a non-zero ``ierr`` / ``info`` instead of an exception where the
reference returns one).  Every numerical call runs on the GPU through
``libadga_b200.so``; nothing here computes the physics on the CPU.
"""
from __future__ import annotations

import ctypes as C
from typing import Dict, Optional

import numpy as np

from . import _lib
from ._lib import ADGA_FP64, ADGA_MIXED, Dims, Outputs, RunStats, Tune, TuneTrial, ptr

PRECISION = {"fp64": ADGA_FP64, "mixed": ADGA_MIXED, ADGA_FP64: ADGA_FP64, ADGA_MIXED: ADGA_MIXED}


class AdgaError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{_lib.ERRORS.get(code, code)}: {msg}")
        self.code = code


def _z(a, shape=None):
    """complex128, Fortran-ordered copy/view with an optional shape check."""
    a = np.asarray(a, dtype=np.complex128)
    if shape is not None and tuple(a.shape) != tuple(shape):
        raise ValueError(f"expected shape {shape}, got {a.shape}")
    return np.asfortranarray(a)


def _i(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.int32))


class Ladder:
    """One resident problem: one-particle data, G(k, nu) table and k-q tables
    on the device (``adga_create``), plus the per-omega vertex store and the
    accumulators of the (q, omega) loop."""

    def __init__(self, *, ndim, nk, nq, iwmax, iwfmax_small, iwbmax_small, beta, mu, iw_data,
                 hk, siw, giw, dc, u, u_tilde, n_dmft, q_data, k_data_eom=None, do_chi=True,
                 do_eom=True, bubble_big_box=False):
        self._lib = _lib.load()
        self.ndim, self.nk, self.nq = ndim, tuple(nk), tuple(nq)
        self.iwmax, self.iwf, self.iwb = iwmax, iwfmax_small, iwbmax_small
        self.beta, self.mu = float(beta), float(mu)
        self.ndim2 = ndim * ndim
        self.maxdim = self.ndim2 * 2 * iwfmax_small
        self.nkp = int(np.prod(nk))
        self.nqp = int(np.prod(nq))
        self.nkp_eom = self.nkp if k_data_eom is None else len(k_data_eom)
        if bubble_big_box and do_chi:
            iwstart, iwstop = -iwmax + iwbmax_small, iwmax - iwbmax_small - 1
        else:
            iwstart, iwstop = -iwfmax_small, iwfmax_small - 1
        self.dims = Dims(ndim, *self.nk, *self.nq, iwmax, iwfmax_small, iwbmax_small, iwstart,
                         iwstop, int(do_chi), int(do_eom), self.nkp_eom, self.beta, self.mu)
        nd, nd2, n2w = ndim, self.ndim2, 2 * iwmax
        self._keep = dict(
            iw=np.ascontiguousarray(np.asarray(iw_data, dtype=np.float64)),
            hk=_z(hk, (nd, nd, self.nkp)), siw=_z(siw, (n2w, nd)), giw=_z(giw, (n2w, nd)),
            dc=_z(dc, (2, nd)), u=_z(u, (nd2, nd2)), ut=_z(u_tilde, (nd2, nd2)),
            nd=_z(n_dmft, (nd,)), q=_i(q_data),
            ke=None if k_data_eom is None else _i(k_data_eom))
        k = self._keep
        h = C.c_void_p()
        rc = self._lib.adga_create(C.byref(self.dims), ptr(k["iw"]), ptr(k["hk"]), ptr(k["siw"]),
                                   ptr(k["giw"]), ptr(k["dc"]), ptr(k["u"]), ptr(k["ut"]),
                                   ptr(k["nd"]), ptr(k["q"]), ptr(k["ke"]), C.byref(h))
        if rc != 0:
            raise AdgaError(rc, "adga_create failed")
        self._h = h
        self.last_npts = 0
        self.last_range = None

    # ------------------------------------------------------------------
    @classmethod
    def from_problem(cls, prob, do_chi=True, do_eom=True, bubble_big_box=False):
        s = prob.spec
        q = generate_q_vol(s.nk, s.nq)
        return cls(ndim=s.ndim, nk=s.nk, nq=s.nq, iwmax=prob.iwmax, iwfmax_small=s.iwf,
                   iwbmax_small=s.iwb, beta=prob.beta, mu=prob.mu, iw_data=prob.iw_data,
                   hk=prob.hk, siw=prob.siw, giw=prob.giw, dc=prob.dc, u=prob.u,
                   u_tilde=prob.u_tilde, n_dmft=prob.n_dmft, q_data=q, do_chi=do_chi,
                   do_eom=do_eom, bubble_big_box=bubble_big_box)

    def close(self):
        if getattr(self, "_h", None):
            self._lib.adga_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, rc, what):
        if rc < 0:
            msg = self._lib.adga_last_error(self._h)
            raise AdgaError(rc, f"{what}: {msg.decode() if msg else ''}")
        return rc

    # ------------------------------------------------------------------
    def device_bytes(self):
        b = C.c_longlong()
        self._check(self._lib.adga_device_bytes(self._h, C.byref(b)), "device_bytes")
        return b.value

    def set_vertex(self, iwb, chi_loc_dens, chi_loc_magn):
        """Stage read_vertex's output for omega = iwb (src/main.F90:525)."""
        N = self.maxdim
        d, m = _z(chi_loc_dens, (N, N)), _z(chi_loc_magn, (N, N))
        self._check(self._lib.adga_set_vertex(self._h, int(iwb), ptr(d), ptr(m)), "set_vertex")

    VERTEX_TYPES = {"full_g4": 0, "connected_g4": 1, "chi_g4": 2}

    def _g4_args(self, vertex_type, g4_dens, g4_magn, ndims):
        vt = self.VERTEX_TYPES[vertex_type] if isinstance(vertex_type, str) else int(vertex_type)
        nd = self.ndim
        W = g4_dens.shape[2] // 2
        shape = (nd, nd, 2 * W, nd, nd, 2 * W)
        d, m = _z(g4_dens, shape), _z(g4_magn, shape)
        nd_arr = np.asfortranarray(np.asarray(ndims if ndims is not None else [[nd, 0]], dtype=np.int32))
        return vt, W, nd_arr, d, m

    def set_vertex_g4(self, iwb, g4_dens, g4_magn, vertex_type="connected_g4", ndims=None):
        """read_vertex (src/hdf5_module.f90:629-773) from the two-particle Green's
        functions g4(ndim, ndim, 2W, ndim, ndim, 2W) as w2dynamics stores them
        (before the beta factor): beta scaling, compound index of the small box
        and the disconnected terms of vertex_type are applied on the GPU, and the
        result is staged like set_vertex.  ndims(nineq, 2): correlated and
        uncorrelated band counts per inequivalent atom (default: one atom, all
        bands correlated)."""
        vt, W, nd_arr, d, m = self._g4_args(vertex_type, g4_dens, g4_magn, ndims)
        self._check(self._lib.adga_set_vertex_g4(self._h, int(iwb), vt, W, nd_arr.shape[0], ptr(nd_arr),
                                                 ptr(d), ptr(m)), "set_vertex_g4")

    def vertex_transform(self, iwb, g4_dens, g4_magn, vertex_type="connected_g4", ndims=None):
        """The same transform, returning (chi_loc_dens, chi_loc_magn), maxdim x maxdim."""
        vt, W, nd_arr, d, m = self._g4_args(vertex_type, g4_dens, g4_magn, ndims)
        N = self.maxdim
        od = np.zeros((N, N), dtype=np.complex128, order="F")
        om = np.zeros((N, N), dtype=np.complex128, order="F")
        self._check(self._lib.adga_vertex_transform(self._h, int(iwb), vt, W, nd_arr.shape[0], ptr(nd_arr),
                                                    ptr(d), ptr(m), ptr(od), ptr(om)), "vertex_transform")
        return od, om

    def _ndims(self, ndims):
        return np.asfortranarray(np.asarray(ndims if ndims is not None else [[self.ndim, 0]], dtype=np.int32))

    def set_threeleg(self, iwb, g3_dens, g3_magn, ndims=None):
        """external_threelegs (src/main.F90:560-561): read_threeleg's transform
        (src/hdf5_module.f90:860-880) of g3(ndim, ndim, ndim, ndim, 2*n3iwf) on
        the GPU; the result replaces gamma^w of omega = iwb."""
        nd = self.ndim
        n3 = np.asarray(g3_dens).shape[4] // 2
        shape = (nd, nd, nd, nd, 2 * n3)
        d, m = _z(g3_dens, shape), _z(g3_magn, shape)
        nd_arr = self._ndims(ndims)
        self._check(self._lib.adga_set_threeleg(self._h, int(iwb), n3, nd_arr.shape[0], ptr(nd_arr),
                                                ptr(d), ptr(m)), "set_threeleg")

    def set_chi_loc_ext(self, chi_dens, chi_magn, ndims=None):
        """external_chi_loc (src/main.F90:407-411): read_chi_loc's transform
        (src/hdf5_module.f90:958-993) of chi(ndim, ndim, ndim, ndim, 2*n2iwb+1)
        on the GPU; the chi_loc outputs are these from now on."""
        nd = self.ndim
        n2 = (np.asarray(chi_dens).shape[4] - 1) // 2
        shape = (nd, nd, nd, nd, 2 * n2 + 1)
        d, m = _z(chi_dens, shape), _z(chi_magn, shape)
        nd_arr = self._ndims(ndims)
        self._check(self._lib.adga_set_chi_loc_ext(self._h, n2, nd_arr.shape[0], ptr(nd_arr), ptr(d), ptr(m)),
                    "set_chi_loc_ext")
        self.ext_chi_loc = True

    def set_vq(self, vq):
        """do_vq: V(q)_{ijkl}, shape (ndim, ndim, ndim, ndim, nqp) in q_data order, as
        read_vq reads it (src/interaction_module.f90:39-123); None switches it off."""
        if vq is None:
            self._check(self._lib.adga_set_vq(self._h, None), "set_vq")
            return
        nd = self.ndim
        v = _z(vq, (nd, nd, nd, nd, self.nqp))
        self._check(self._lib.adga_set_vq(self._h, ptr(v)), "set_vq")

    def reset_outputs(self):
        self._check(self._lib.adga_reset_outputs(self._h), "reset_outputs")

    def ladder_run(self, qwstart=1, qwstop=None, precision="fp64"):
        """The (q, omega) loop of src/main.F90:486-799 over compound points
        qwstart..qwstop (1-based, omega outer).  Returns (status, stats)."""
        if qwstop is None:
            qwstop = self.nqp * (2 * self.iwb + 1)
        n = qwstop - qwstart + 1
        status = np.zeros(n, dtype=np.int32)
        st = RunStats()
        rc = self._lib.adga_ladder_run(self._h, int(qwstart), int(qwstop), PRECISION[precision],
                                       status.ctypes.data_as(C.POINTER(C.c_int)), C.byref(st))
        self._check(rc, "ladder_run")
        self.last_npts = n
        self.last_range = (qwstart, qwstop)
        return status, st.as_dict()

    # ---- kernel choices of the mixed path ------------------------------
    @property
    def tune(self) -> Dict[str, int]:
        """The mixed path's kernel choices (adga_get_tune): factor (0: FP32 LU
        + FP64 refinement, 1: FP64 LU), pairs (0: one tensor-core update per
        step, 1: delayed pairs, 2: groups of three, 3: groups of four), tri_tc,
        batch, resid, trsv_tc."""
        t = Tune()
        self._check(self._lib.adga_get_tune(self._h, C.byref(t)), "get_tune")
        return t.as_dict()

    @tune.setter
    def tune(self, cfg: Dict[str, int]):
        t = Tune(**{**self.tune, **cfg})
        self._check(self._lib.adga_set_tune(self._h, C.byref(t)), "set_tune")

    def autotune(self, qwstart, qwstop, tol=1e-8):
        """Measure the mixed path's configurations on points qwstart..qwstop
        against the FP64 path and keep the fastest one within tol
        (adga_autotune; resets the accumulators).  Returns (choice, trials)."""
        trials = (TuneTrial * 16)()
        n = C.c_int()
        best = Tune()
        self._check(self._lib.adga_autotune(self._h, int(qwstart), int(qwstop), float(tol), trials, 16,
                                            C.byref(n), C.byref(best)), "autotune")
        out = [dict(**trials[i].tune.as_dict(), ms=trials[i].ms, err=trials[i].err,
                    accepted=bool(trials[i].accepted)) for i in range(n.value)]
        return best.as_dict(), out

    def output_shapes(self, npts=None) -> Dict[str, tuple]:
        """Shapes of the accumulators get_outputs returns (npts: points of the run)."""
        nd, nd2, nw = self.ndim, self.ndim2, 2 * self.iwb + 1
        n = self.last_npts if npts is None else npts
        return dict(chi_qw_dens=(nd2, nd2, n), chi_qw_magn=(nd2, nd2, n), bubble_nl=(nd2, nd2, n),
                    bubble_loc=(nd2, nd2, nw), chi_loc_dens=(nd2, nd2, nw), chi_loc_magn=(nd2, nd2, nw),
                    sigma_nl=(nd, nd, 2 * self.iwf, self.nkp_eom), sigma_dmft=(nd, nd, 2 * self.iwf),
                    sigma_hf=(nd, nd, self.nkp_eom))

    def get_outputs(self, out: Dict[str, np.ndarray] = None) -> Dict[str, np.ndarray]:
        """Accumulators with the reference's shapes (Fortran order):
        chi_qw_dens/magn, bubble_nl (ndim2, ndim2, npts); bubble_loc,
        chi_loc_dens/magn (ndim2, ndim2, 2*iwb+1); sigma_nl
        (ndim, ndim, 2*iwf, nkp_eom); sigma_dmft (ndim, ndim, 2*iwf);
        sigma_hf (ndim, ndim, nkp_eom).  `out`: caller-owned arrays of these
        shapes (complex128, Fortran order; pinned host memory makes the copies
        fastest) to fill instead of new ones."""
        shapes = self.output_shapes()
        if out is None:
            out = {k: np.zeros(sh, dtype=np.complex128, order="F") for k, sh in shapes.items()}
        else:
            for k, sh in shapes.items():
                a = out[k]
                if a.shape != sh or a.dtype != np.complex128 or not a.flags.f_contiguous:
                    raise ValueError(f"out[{k!r}]: expected complex128 {sh} in Fortran order")
        o = Outputs(*[out[k].ctypes.data for k, _ in Outputs._fields_])
        self._check(self._lib.adga_get_outputs(self._h, C.byref(o)), "get_outputs")
        return out

    # ---- derivatives (forward-mode tangents) ------------------------------
    def set_tangent(self, dhk=None, du=None, du_tilde=None, direction=0):
        """Input tangents of parameter direction `direction` (0..3): dH(k)
        (ndim, ndim, nkp), du and du_tilde (ndim2, ndim2); None = zero."""
        nd, nd2 = self.ndim, self.ndim2
        a = None if dhk is None else _z(dhk, (nd, nd, self.nkp))
        b = None if du is None else _z(du, (nd2, nd2))
        c = None if du_tilde is None else _z(du_tilde, (nd2, nd2))
        self._check(self._lib.adga_set_tangent(self._h, int(direction), ptr(a), ptr(b), ptr(c)), "set_tangent")

    def set_vertex_tangent(self, iwb, dchi_loc_dens, dchi_loc_magn, direction=0):
        """dchi_loc^{dens,magn}(omega = iwb) of a direction (None clears it)."""
        if dchi_loc_dens is None:
            self._check(self._lib.adga_set_vertex_tangent(self._h, int(direction), int(iwb), None, None),
                        "set_vertex_tangent")
            return
        N = self.maxdim
        d, m = _z(dchi_loc_dens, (N, N)), _z(dchi_loc_magn, (N, N))
        self._check(self._lib.adga_set_vertex_tangent(self._h, int(direction), int(iwb), ptr(d), ptr(m)),
                    "set_vertex_tangent")

    def clear_tangents(self):
        self._check(self._lib.adga_clear_tangents(self._h), "clear_tangents")

    def ladder_run_tangent(self, qwstart=1, qwstop=None, precision="fp64"):
        """The ladder (FP64 or mixed) plus the tangents of every direction set before."""
        if qwstop is None:
            qwstop = self.nqp * (2 * self.iwb + 1)
        n = qwstop - qwstart + 1
        status = np.zeros(n, dtype=np.int32)
        st = RunStats()
        rc = self._lib.adga_ladder_run_tangent(self._h, int(qwstart), int(qwstop), PRECISION[precision],
                                               status.ctypes.data_as(C.POINTER(C.c_int)), C.byref(st))
        self._check(rc, "ladder_run_tangent")
        self.last_npts = n
        self.last_range = (qwstart, qwstop)
        return status, st.as_dict()

    def get_tangent_outputs(self, direction=0) -> Dict[str, np.ndarray]:
        """Tangents of the accumulators of one direction, shapes as get_outputs."""
        nd, nd2, nw, n = self.ndim, self.ndim2, 2 * self.iwb + 1, self.last_npts
        z = lambda *s: np.zeros(s, dtype=np.complex128, order="F")
        out = dict(chi_qw_dens=z(nd2, nd2, n), chi_qw_magn=z(nd2, nd2, n), bubble_nl=z(nd2, nd2, n),
                   bubble_loc=z(nd2, nd2, nw), chi_loc_dens=z(nd2, nd2, nw),
                   chi_loc_magn=z(nd2, nd2, nw), sigma_nl=z(nd, nd, 2 * self.iwf, self.nkp_eom),
                   sigma_dmft=z(nd, nd, 2 * self.iwf), sigma_hf=z(nd, nd, self.nkp_eom))
        o = Outputs(*[out[k].ctypes.data for k, _ in Outputs._fields_])
        self._check(self._lib.adga_get_tangent_outputs(self._h, int(direction), C.byref(o)), "get_tangent_outputs")
        return out

    def assemble_tangent(self, dout):
        """Tangents of the assembled chi(q, w) and Sigma (siw is held fixed)."""
        zero_siw = np.zeros((2 * self.iwmax, self.ndim), complex)
        return self.assemble(dout, zero_siw)

    def assemble(self, out, siw):
        """chi(q,w) = chi_nl + bubble_nl + chi_loc(w) (with chi_loc += bubble_loc)
        and Sigma = Sigma_nl + siw (src/main.F90:935-936,1050-1063,1127-1140;
        add_siw_dmft, src/eom_module.f90:237-251)."""
        qs, _ = self.last_range
        widx = (np.arange(qs, qs + self.last_npts) - 1) // self.nqp
        if getattr(self, "ext_chi_loc", False):     # external chi_loc holds the bubble already
            cld, clm = out["chi_loc_dens"], out["chi_loc_magn"]
        else:
            cld = out["chi_loc_dens"] + out["bubble_loc"]
            clm = out["chi_loc_magn"] + out["bubble_loc"]
        chi_d = out["chi_qw_dens"] + out["bubble_nl"] + cld[:, :, widx]
        chi_m = out["chi_qw_magn"] + out["bubble_nl"] + clm[:, :, widx]
        sig = out["sigma_nl"].copy(order="F")
        nu = np.arange(-self.iwf, self.iwf) + self.iwmax
        for b in range(self.ndim):
            sig[b, b] += np.asarray(siw)[nu, b][:, None]
        return dict(chi_dens=chi_d, chi_magn=chi_m, chi_loc_dens=cld, chi_loc_magn=clm, sigma=sig)

    def post_loop(self, sigma_sum=None, want=("sigma_loc", "gloc", "n_dga_k", "n_dga")):
        """Post-loop assembly of src/main.F90:869-890 on the GPU: add_siw_dmft,
        get_sigma_g_loc (full k mesh only) and get_ndga.  sigma_sum: the reduced
        non-local self-energy (ndim, ndim, 2*iwf, nkp_eom); None uses this
        handle's own accumulated Sigma_nl.  Returns a dict with 'sigma_sum'
        (Sigma_nl + siw) and the requested outputs."""
        nd, iwf = self.ndim, self.iwf
        nke = self.nkp_eom
        sig = (np.zeros((nd, nd, 2 * iwf, nke), dtype=np.complex128, order="F") if sigma_sum is None
               else _z(sigma_sum, (nd, nd, 2 * iwf, nke)).copy(order="F"))
        bufs = {"sigma_loc": (nd, nd, 2 * iwf), "gloc": (2 * self.iwmax, nd, nd),
                "n_dga_k": (nke, nd, nd), "n_dga": (nd,)}
        out = {k: np.zeros(v, dtype=np.complex128, order="F") for k, v in bufs.items() if k in want}
        self._check(self._lib.adga_post_loop(self._h, ptr(sig) if sigma_sum is not None else None,
                                             ptr(out.get("sigma_loc")), ptr(out.get("gloc")),
                                             ptr(out.get("n_dga_k")), ptr(out.get("n_dga"))), "post_loop")
        if sigma_sum is not None:
            out["sigma_sum"] = sig
        return out

    # ---- per-routine entry points -------------------------------------
    def get_chi0_loc(self, iwf, iwb):
        out = np.zeros((self.ndim2, self.ndim2), dtype=np.complex128, order="F")
        self._check(self._lib.adga_get_chi0_loc(self._h, int(iwf), int(iwb), ptr(out)), "get_chi0_loc")
        return out

    def get_chi0_loc_inv(self, iwf, iwb):
        out = np.zeros((self.ndim2, self.ndim2), dtype=np.complex128, order="F")
        self._check(self._lib.adga_get_chi0_loc_inv(self._h, int(iwf), int(iwb), ptr(out)),
                    "get_chi0_loc_inv")
        return out

    def chi0_q(self, iq, iwb):
        """(chi0q(ndim2, ndim2, 2*iwf), bubble_nl) at 1-based iq (src/main.F90:644-663)."""
        c = np.zeros((self.ndim2, self.ndim2, 2 * self.iwf), dtype=np.complex128, order="F")
        b = np.zeros((self.ndim2, self.ndim2), dtype=np.complex128, order="F")
        self._check(self._lib.adga_chi0_q(self._h, int(iq), int(iwb), ptr(c), ptr(b)), "chi0_q")
        return c, b

    def bse_point(self, iq, iwb, precision="fp64"):
        """(etaqd, etaqm, gammaqd, info) of src/main.F90:674-757 at 1-based iq."""
        sh = (self.ndim2, self.maxdim)
        ed, em, gq = (np.zeros(sh, dtype=np.complex128, order="F") for _ in range(3))
        info = C.c_int()
        rc = self._lib.adga_bse_point(self._h, int(iq), int(iwb), PRECISION[precision], ptr(ed),
                                      ptr(em), ptr(gq), C.byref(info))
        self._check(rc, "bse_point")
        return ed, em, gq, info.value

    def get_gamma_w(self, iwb):
        sh = (self.ndim2, self.maxdim)
        gd, gm = (np.zeros(sh, dtype=np.complex128, order="F") for _ in range(2))
        self._check(self._lib.adga_get_gamma_w(self._h, int(iwb), ptr(gd), ptr(gm)), "get_gamma_w")
        return gd, gm

    def calc_chi_qw(self, chi_qw, interm3, chi0_sum):
        """chi_qw += beta^-2 sum interm3 chi0_sum, in place (src/susc_module.f90:34-56)."""
        if not (isinstance(chi_qw, np.ndarray) and chi_qw.dtype == np.complex128 and chi_qw.flags.f_contiguous):
            raise ValueError("chi_qw must be a Fortran-ordered complex128 array (updated in place)")
        i3 = _z(interm3, (self.ndim2, self.maxdim))
        c0 = _z(chi0_sum, (self.ndim2, self.ndim2, 2 * self.iwf))
        self._check(self._lib.adga_calc_chi_qw(self._h, ptr(chi_qw), ptr(i3), ptr(c0)), "calc_chi_qw")
        return chi_qw

    def calc_eom_dynamic(self, etaqd, etaqm, gammaqd, iwb, iq, sigma_nl):
        sh = (self.ndim2, self.maxdim)
        ed, em, gq = _z(etaqd, sh), _z(etaqm, sh), _z(gammaqd, sh)
        if not (sigma_nl.dtype == np.complex128 and sigma_nl.flags.f_contiguous):
            raise ValueError("sigma_nl must be Fortran-ordered complex128 (updated in place)")
        self._check(self._lib.adga_calc_eom_dynamic(self._h, ptr(ed), ptr(em), ptr(gq), int(iwb),
                                                    int(iq), ptr(sigma_nl)), "calc_eom_dynamic")
        return sigma_nl

    def calc_eom_dmft(self, gammawd, iwb, sigma_dmft):
        g = _z(gammawd, (self.ndim2, self.maxdim))
        self._check(self._lib.adga_calc_eom_dmft(self._h, ptr(g), int(iwb), ptr(sigma_dmft)),
                    "calc_eom_dmft")
        return sigma_dmft

    def calc_eom_static(self, iq, sigma_dmft):
        self._check(self._lib.adga_calc_eom_static(self._h, int(iq), ptr(sigma_dmft)),
                    "calc_eom_static")
        return sigma_dmft


# ---- standalone routines ---------------------------------------------------
def inverse_matrix(M):
    """GPU inverse of a square complex matrix: (Minv, ierr, erstr) like
    inverse_matrix_z (src/lapack_module.f90:40-70)."""
    lib = _lib.load()
    A = np.array(M, dtype=np.complex128, order="F", copy=True)
    n = A.shape[0]
    if A.shape != (n, n):
        raise ValueError("square matrix expected")
    ierr = C.c_int()
    buf = C.create_string_buffer(200)
    rc = lib.adga_inverse_matrix_z(ptr(A), n, C.byref(ierr), buf)
    if rc < 0:
        raise AdgaError(rc, "inverse_matrix_z")
    return A, ierr.value, buf.value.decode()


def index2component_band(nbands, ind):
    """index2component_band (src/aux.f90:169-186): 1-based band pattern of a
    1-based vertex group index."""
    lib = _lib.load()
    b = np.zeros(4, dtype=np.int32)
    rc = lib.adga_index2component_band(int(nbands), int(ind), ptr(b))
    if rc:
        raise AdgaError(rc, "index2component_band: index out of range")
    return tuple(int(x) for x in b)


def generate_q_vol(nk, nq):
    lib = _lib.load()
    q = np.zeros(int(np.prod(nq)), dtype=np.int32)
    rc = lib.adga_generate_q_vol(*map(int, nk), *map(int, nq), ptr(q))
    if rc:
        raise AdgaError(rc, "generate_q_vol: mismatch between k- and q-grid")
    return q


def index_kq(nk, q_data, k_sel=None):
    """ind(k, q) = k - q (1-based, Fortran order (nk_sel, nqp)); index_kq / index_kq_eom."""
    lib = _lib.load()
    q = _i(q_data)
    ks = None if k_sel is None else _i(k_sel)
    nks = int(np.prod(nk)) if ks is None else len(ks)
    ind = np.zeros((nks, len(q)), dtype=np.int32, order="F")
    rc = lib.adga_index_kq(*map(int, nk), ptr(q), len(q), ptr(ks), nks, ptr(ind))
    if rc:
        raise AdgaError(rc, "index_kq")
    return ind


def create_u(ndim, U, V, J):
    """Kanamori (Umat, u, u_tilde) for one atom of correlated bands (create_u)."""
    lib = _lib.load()
    nd2 = ndim * ndim
    Um = np.zeros((ndim,) * 4, order="F")
    u = np.zeros((nd2, nd2), dtype=np.complex128, order="F")
    ut = np.zeros_like(u)
    rc = lib.adga_create_u(int(ndim), float(U), float(V), float(J), ptr(Um), ptr(u), ptr(ut))
    if rc:
        raise AdgaError(rc, "create_u")
    return Um, u, ut


def run_ladder(prob, precision="fp64", qwstart=1, qwstop=None, do_chi=True, do_eom=True,
               bubble_big_box=False):
    """Convenience driver: stage every needed vertex, run, return outputs."""
    s = prob.spec
    lad = Ladder.from_problem(prob, do_chi=do_chi, do_eom=do_eom, bubble_big_box=bubble_big_box)
    try:
        nqp = s.nqp
        qwstop = nqp * (2 * s.iwb + 1) if qwstop is None else qwstop
        for iwb in sorted({-s.iwb + (i - 1) // nqp for i in range(qwstart, qwstop + 1)}):
            d, m = prob.vertex(iwb)
            lad.set_vertex(iwb, d, m)
        status, stats = lad.ladder_run(qwstart, qwstop, precision)
        out = lad.get_outputs()
        out.update(lad.assemble(out, prob.siw))
        out["status"], out["stats"] = status, stats
        return out
    finally:
        lad.close()
