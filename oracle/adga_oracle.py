"""NumPy/SciPy restatement of the ADGA per-(q, omega) ladder hot path.

TEST INFRASTRUCTURE ONLY -- this is the FP64 oracle the CUDA path is checked
against.  It is never imported by the product package ``adga_b200``.

Every routine follows one reference routine (paths relative to the reference
project root) and keeps its index conventions:

* arrays carry the reference's Fortran shapes with 0-based Python indices and
  Fortran (column-major) memory order, e.g. ``hk[i, j, ik]`` is
  ``hk(i+1, j+1, ik+1)``; frequency axes are shifted so that index
  ``n + iwmax`` holds Matsubara index ``n``;
* orbital compound indices are the reference's: ``{i,j} -> i*ndim + j`` for the
  row index of chi0 (``src/one_particle_quant_module.f90:274-288``) and
  ``{l,k} -> l*ndim + k`` for its column; the big BSE index is
  ``i2 + dum*ndim2`` with ``dum = iwf + iwfmax_small``
  (``src/main.F90:546``).

Parity status: UNPINNED against the Fortran binary (it cannot be built in this
image); ``create_u`` is pinned against ``documentation/examples/umatrix`` and
``read_hk`` against ``srvo3-testdata/srvo3_k20.hk``; everything else is pinned
by the analytic known-answer tests in ``tests/test_oracle.py``.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Callable, Dict, Optional, Sequence, Tuple

import numpy as np
from scipy.linalg import lapack

CI = 1j


# --------------------------------------------------------------------------
# k / q grid tools -- src/kq_tools.f90
# --------------------------------------------------------------------------
def k_vector(ik, nk):
    """1-based linear index -> integer (kx, ky, kz); src/kq_tools.f90:137-144."""
    nkpx, nkpy, nkpz = nk
    ik = np.asarray(ik)
    kz = (ik - 1) % nkpz
    ky = ((ik - 1) // nkpz) % nkpy
    kx = (ik - 1) // (nkpy * nkpz)
    return kx, ky, kz


def k_index(kx, ky, kz, nk):
    """Integer coords -> 1-based linear index (kz fastest); src/kq_tools.f90:119-125."""
    nkpx, nkpy, nkpz = nk
    return 1 + np.asarray(kz) + np.asarray(ky) * nkpz + np.asarray(kx) * nkpy * nkpz


def k_minus_q(ik, iq, nk):
    """Index of k - q with per-axis modulo fold-back; src/kq_tools.f90:96-108."""
    nkpx, nkpy, nkpz = nk
    ix, iy, iz = k_vector(ik, nk)
    lx, ly, lz = k_vector(iq, nk)
    return (1 + (nkpz + iz - lz) % nkpz + ((nkpy + iy - ly) % nkpy) * nkpz
            + ((nkpx + ix - lx) % nkpx) * nkpy * nkpz)


def generate_q_vol(nk, nq):
    """q-grid as the subset q_i = i*nk/nq of the k-grid; src/kq_tools.f90:42-57."""
    nkpx, nkpy, nkpz = nk
    nqpx, nqpy, nqpz = nq
    out = []
    for i in range(nqpx):
        for j in range(nqpy):
            for k in range(nqpz):
                out.append(int(k_index(i * nkpx // nqpx, j * nkpy // nqpy,
                                       k * nkpz // nqpz, nk)))
    return np.array(out, dtype=np.int32)


def index_kq(nk, q_data, k_data=None):
    """ind(ik, iq) = k_minus_q(k, q) (1-based); src/kq_tools.f90:59-85."""
    nkp = nk[0] * nk[1] * nk[2]
    ks = np.arange(1, nkp + 1) if k_data is None else np.asarray(k_data)
    ind = np.zeros((len(ks), len(q_data)), dtype=np.int32, order="F")
    for jq, q in enumerate(q_data):
        ind[:, jq] = k_minus_q(ks, q, nk)
    return ind


# --------------------------------------------------------------------------
# interaction -- src/interaction_module.f90:182-291 and src/aux.f90:157-286
# --------------------------------------------------------------------------
def _index2cor(ndims, m, n, o, p):
    a = b = c = d = 0
    for ineq in range(1, len(ndims) + 1):
        dimstart = 1
        for i in range(2, ineq + 1):
            dimstart += ndims[i - 2][0] + ndims[i - 2][1]
        dimend = dimstart + ndims[ineq - 1][0] - 1
        if dimstart <= m <= dimend: a = ineq
        if dimstart <= n <= dimend: b = ineq
        if dimstart <= o <= dimend: c = ineq
        if dimstart <= p <= dimend: d = ineq
    return a == b and c == d and a == d and a != 0


def _index2uncor(ndims, m, n, o, p):
    a = b = c = d = 0
    for ineq in range(1, len(ndims) + 1):
        dimstart = ndims[0][0] + 1
        for i in range(2, ineq + 1):
            dimstart += ndims[i - 1][0] + ndims[i - 2][1]
        dimend = dimstart + ndims[ineq - 1][1] - 1
        if dimstart <= m <= dimend: a = ineq
        if dimstart <= n <= dimend: b = ineq
        if dimstart <= o <= dimend: c = ineq
        if dimstart <= p <= dimend: d = ineq
    return a == b and c == d and a == d and a != 0


def _index2ineq(ndims, m, n, o, p):
    a = b = c = d = 0
    for ineq in range(1, len(ndims) + 1):
        dimstart = 1
        for i in range(2, ineq + 1):
            dimstart += ndims[i - 2][0] + ndims[i - 2][1]
        dimend = dimstart + ndims[ineq - 1][0] + ndims[ineq - 1][1] - 1
        if dimstart <= m <= dimend: a = ineq
        if dimstart <= n <= dimend: b = ineq
        if dimstart <= o <= dimend: c = ineq
        if dimstart <= p <= dimend: d = ineq
    return a if (a == b and c == d and a == d) else 0


def component2index_band(nbands, b1, b2, b3, b4):
    """src/aux.f90:157-164 (1-based bands and group index)."""
    return nbands ** 3 * (b1 - 1) + nbands ** 2 * (b2 - 1) + nbands * (b3 - 1) + b4


def index2component_band(nbands, ind):
    """src/aux.f90:169-186 (1-based group index -> 1-based bands)."""
    it = ind - 1
    n3, n2 = nbands ** 3, nbands ** 2
    b1 = it // n3 + 1
    b2 = (it - n3 * (b1 - 1)) // n2 + 1
    b3 = (it - n3 * (b1 - 1) - n2 * (b2 - 1)) // nbands + 1
    b4 = it - n3 * (b1 - 1) - n2 * (b2 - 1) - nbands * (b3 - 1) + 1
    return b1, b2, b3, b4


FULL_G4, CONNECTED_G4, CHI_G4 = 0, 1, 2   # src/parameters_module.f90:74


def read_vertex_transform(g4_dens, g4_magn, iwb, vertex_type, ndims, giw, beta, iwf, iwmax):
    """The compound-index part of read_vertex (src/hdf5_module.f90:700,711 and
    :718-770): g4(ndim, ndim, 2W, ndim, ndim, 2W) as w2dynamics stores it
    (index n + W holds Matsubara n, before the beta factor) -> chi_loc of the
    small box (maxdim x maxdim) with the disconnected terms of vertex_type.
    giw[n + iwmax, i] is the local Green's function."""
    nd = g4_dens.shape[0]
    W = g4_dens.shape[2] // 2
    nd2 = nd * nd
    N = nd2 * 2 * iwf
    g4d = np.asarray(g4_dens) * beta
    g4m = np.asarray(g4_magn) * beta
    cd = np.zeros((N, N), complex)
    cm = np.zeros((N, N), complex)
    cor = {}
    for i in range(nd):
        for j in range(nd):
            for k in range(nd):
                for l in range(nd):
                    cor[i, j, k, l] = _index2cor(ndims, i + 1, j + 1, k + 1, l + 1)
    g = lambda n, b: giw[n + iwmax, b]
    i2 = 0
    for w2 in range(-iwf, iwf):
        for l in range(nd):
            for k in range(nd):
                i1 = 0
                for w1 in range(-iwf, iwf):
                    for i in range(nd):
                        for j in range(nd):
                            cm[i1, i2] = g4m[i, j, w1 + W, k, l, w2 + W]
                            cd[i1, i2] = g4d[i, j, w1 + W, k, l, w2 + W]
                            c4 = cor[i, j, k, l]
                            bub = w2 == w1 and i == l and j == k
                            if vertex_type == FULL_G4:
                                if iwb == 0 and i == j and k == l and c4:
                                    cd[i1, i2] -= 2.0 * beta * g(w1, i) * g(w2, l)
                                if bub and not c4:
                                    t = beta * g(w1, i) * g(w2 - iwb, j)
                                    cd[i1, i2] -= t
                                    cm[i1, i2] -= t
                            elif vertex_type == CONNECTED_G4:
                                if bub:
                                    t = beta * g(w1, i) * g(w2 - iwb, j)
                                    cd[i1, i2] -= t
                                    cm[i1, i2] -= t
                            elif vertex_type == CHI_G4:
                                if bub and not c4:
                                    t = beta * g(w1, i) * g(w2 - iwb, j)
                                    cd[i1, i2] -= t
                                    cm[i1, i2] -= t
                            i1 += 1
                i2 += 1
    return np.asfortranarray(cd), np.asfortranarray(cm)


def create_u(ndims, Udd, Vdd, Jdd, Upp=None, Vpp=None, Jpp=None,
             Udp=None, Vdp=None, Jdp=None, interaction_mode=None):
    """Kanamori/density-density U tensor and its compound forms.

    Restates ``create_u`` (src/interaction_module.f90:182-291).  ``ndims`` is
    the list of (n_correlated, n_uncorrelated) bands per inequivalent atom;
    the per-atom parameter lists follow the reference's Udd/Vdd/Jdd/... arrays.
    Returns (Umat[ndim]^4, u[ndim2, ndim2], u_tilde[ndim2, ndim2]) with
    u({k,i},{j,l}) = U_ijkl and u_tilde({k,i},{j,l}) = U_ijlk.
    """
    nineq = len(ndims)
    z = [0.0] * nineq
    Upp = Upp or z; Vpp = Vpp or z; Jpp = Jpp or z
    Udp = Udp or z; Vdp = Vdp or z; Jdp = Jdp or z
    mode = interaction_mode or [1] * nineq
    ndim = sum(a + b for a, b in ndims)
    Umat = np.zeros((ndim, ndim, ndim, ndim), order="F")
    for i in range(1, ndim + 1):
        for j in range(1, ndim + 1):
            for k in range(1, ndim + 1):
                for l in range(1, ndim + 1):
                    ineq = _index2ineq(ndims, i, j, k, l)
                    if ineq == 0:
                        continue
                    e = ineq - 1
                    if _index2cor(ndims, i, j, k, l):
                        UU, VV, JJ = Udd[e], Vdd[e], Jdd[e]
                    elif _index2uncor(ndims, i, j, k, l):
                        UU, VV, JJ = Upp[e], Vpp[e], Jpp[e]
                    else:
                        UU, VV, JJ = Udp[e], Vdp[e], Jdp[e]
                    val = None
                    if i == j and k == l:
                        if i == k:
                            val = UU
                        elif mode[e] == 1:
                            val = JJ
                    if val is None and i == k and j == l:
                        val = VV
                    if val is None and i == l and j == k and mode[e] == 1:
                        val = JJ
                    if val is not None:
                        Umat[i - 1, j - 1, k - 1, l - 1] = val
    nd2 = ndim * ndim
    u = np.zeros((nd2, nd2), dtype=complex, order="F")
    ut = np.zeros((nd2, nd2), dtype=complex, order="F")
    for l in range(ndim):
        for j in range(ndim):
            i2 = l * ndim + j
            for i in range(ndim):
                for k in range(ndim):
                    i1 = i * ndim + k
                    u[i1, i2] = Umat[i, j, k, l]
                    ut[i1, i2] = Umat[i, j, l, k]
    return Umat, u, ut


def read_umatrix(path, ndim):
    """Text U-matrix reader (src/interaction_module.f90:128-177)."""
    Umat = np.zeros((ndim,) * 4, order="F")
    with open(path) as fh:
        fh.readline()
        for _ in range(ndim ** 4):
            parts = fh.readline().split()
            i, j, k, l = (int(x) for x in parts[:4])
            Umat[i - 1, j - 1, k - 1, l - 1] = float(parts[4])
    return Umat


# --------------------------------------------------------------------------
# .hk text format -- src/hdf5_module.f90:339-378
# --------------------------------------------------------------------------
def read_hk(path):
    """Return (k_data[3, nkp], hk[ndim, ndim, nkp]) from a w2w ``.hk`` file."""
    with open(path) as fh:
        toks = fh.read().split("\n")
    head = toks[0].split()
    nkp, ndim = int(head[0]), int(head[1])
    hk = np.zeros((ndim, ndim, nkp), dtype=complex, order="F")
    kd = np.zeros((3, nkp), order="F")
    pos = 1
    for ik in range(nkp):
        kd[:, ik] = [float(x) for x in toks[pos].split()[:3]]
        pos += 1
        for i in range(ndim):
            v = [float(x) for x in toks[pos].split()]
            pos += 1
            hk[i, :, ik] = np.array(v[0::2][:ndim]) + CI * np.array(v[1::2][:ndim])
    return kd, hk


# --------------------------------------------------------------------------
# small closed-form inverses -- src/aux.f90:288-325
# --------------------------------------------------------------------------
def inverse_matrix_3(A):
    """Cofactor inverse of a stack (..., 3, 3); same algebra as the reference."""
    a = A
    detinv = 1.0 / (a[..., 0, 0] * a[..., 1, 1] * a[..., 2, 2] - a[..., 0, 0] * a[..., 1, 2] * a[..., 2, 1]
                    - a[..., 0, 1] * a[..., 1, 0] * a[..., 2, 2] + a[..., 0, 1] * a[..., 1, 2] * a[..., 2, 0]
                    + a[..., 0, 2] * a[..., 1, 0] * a[..., 2, 1] - a[..., 0, 2] * a[..., 1, 1] * a[..., 2, 0])
    B = np.empty_like(a)
    B[..., 0, 0] = +detinv * (a[..., 1, 1] * a[..., 2, 2] - a[..., 1, 2] * a[..., 2, 1])
    B[..., 1, 0] = -detinv * (a[..., 1, 0] * a[..., 2, 2] - a[..., 1, 2] * a[..., 2, 0])
    B[..., 2, 0] = +detinv * (a[..., 1, 0] * a[..., 2, 1] - a[..., 1, 1] * a[..., 2, 0])
    B[..., 0, 1] = -detinv * (a[..., 0, 1] * a[..., 2, 2] - a[..., 0, 2] * a[..., 2, 1])
    B[..., 1, 1] = +detinv * (a[..., 0, 0] * a[..., 2, 2] - a[..., 0, 2] * a[..., 2, 0])
    B[..., 2, 1] = -detinv * (a[..., 0, 0] * a[..., 2, 1] - a[..., 0, 1] * a[..., 2, 0])
    B[..., 0, 2] = +detinv * (a[..., 0, 1] * a[..., 1, 2] - a[..., 0, 2] * a[..., 1, 1])
    B[..., 1, 2] = -detinv * (a[..., 0, 0] * a[..., 1, 2] - a[..., 0, 2] * a[..., 1, 0])
    B[..., 2, 2] = +detinv * (a[..., 0, 0] * a[..., 1, 1] - a[..., 0, 1] * a[..., 1, 0])
    return B


def inverse_matrix_2(A):
    detinv = 1.0 / (A[..., 0, 0] * A[..., 1, 1] - A[..., 0, 1] * A[..., 1, 0])
    B = np.empty_like(A)
    B[..., 0, 0] = +detinv * A[..., 1, 1]
    B[..., 1, 0] = -detinv * A[..., 1, 0]
    B[..., 0, 1] = -detinv * A[..., 0, 1]
    B[..., 1, 1] = +detinv * A[..., 0, 0]
    return B


def inverse_matrix(M):
    """zgetrf + zgetri, as ``inverse_matrix_z`` (src/lapack_module.f90:40-70).

    Returns (inverse, ierr, erstr) with the reference's error strings.
    """
    lu, piv, info = lapack.zgetrf(np.asfortranarray(M))
    if info != 0:
        return lu, int(info), "ERROR in ZGETRF"
    inv, info = lapack.zgetri(lu, piv)
    if info != 0:
        return inv, int(info), "ERROR in ZGETRI"
    return inv, 0, ""


# --------------------------------------------------------------------------
# inputs
# --------------------------------------------------------------------------
@dataclass
class LadderInputs:
    """All implicit globals of the hot path (src/parameters_module.f90:43-101)."""
    ndim: int
    nk: Tuple[int, int, int]
    nq: Tuple[int, int, int]
    iwmax: int
    iwfmax_small: int
    iwbmax_small: int
    beta: float
    mu: float
    hk: np.ndarray          # (ndim, ndim, nkp) complex, F-order
    siw: np.ndarray         # (2*iwmax, ndim) complex: index n+iwmax
    giw: np.ndarray         # (2*iwmax, ndim) complex
    dc: np.ndarray          # (2, ndim) complex
    u: np.ndarray           # (ndim2, ndim2) complex
    u_tilde: np.ndarray     # (ndim2, ndim2) complex
    n_dmft: np.ndarray      # (ndim,) complex
    vertex: Callable[[int], Tuple[np.ndarray, np.ndarray]]  # iwb -> (chi_d, chi_m)
    do_chi: bool = True
    do_eom: bool = True
    bubble_big_box: bool = False  # "[Debug] Bubble" (src/config_module.f90:467-477)
    iw_data: Optional[np.ndarray] = None
    # external_threelegs: iwb -> (gamma_d, gamma_m) (ndim2, maxdim) as read_threeleg
    # returns them (src/main.F90:560-561); None = gamma^w from F~ (:563-570)
    threeleg: Optional[Callable[[int], Tuple[np.ndarray, np.ndarray]]] = None
    # external_chi_loc: (chi_loc_dens, chi_loc_magn) (ndim2, ndim2, 2*iwb+1) as
    # read_chi_loc returns them (src/main.F90:407-411); None = built from gamma^w
    chi_loc_ext: Optional[Tuple[np.ndarray, np.ndarray]] = None
    # do_vq: V(q) per q point, (ndim2, ndim2, nqp) as read_vq returns it
    # (src/interaction_module.f90:39-123); None = no non-local interaction
    vq: Optional[np.ndarray] = None

    def __post_init__(self):
        if self.iw_data is None:
            n = np.arange(-self.iwmax, self.iwmax)
            self.iw_data = np.pi * (2 * n + 1) / self.beta

    @property
    def ndim2(self): return self.ndim * self.ndim
    @property
    def maxdim(self): return self.ndim2 * 2 * self.iwfmax_small
    @property
    def nkp(self): return self.nk[0] * self.nk[1] * self.nk[2]
    @property
    def nqp(self): return self.nq[0] * self.nq[1] * self.nq[2]
    @property
    def iw_range(self):
        """(iwstart, iwstop) of the chi0 nu-sum; src/config_module.f90:467-477."""
        if self.bubble_big_box and self.do_chi:
            return -self.iwmax + self.iwbmax_small, self.iwmax - self.iwbmax_small - 1
        return -self.iwfmax_small, self.iwfmax_small - 1


class Oracle:
    """The reference's hot path, one (q, omega) point at a time."""

    def __init__(self, inp: LadderInputs):
        self.inp = inp
        self.q_data = generate_q_vol(inp.nk, inp.nq)
        self.kq_ind = index_kq(inp.nk, self.q_data)      # 1-based
        self._gk_cache: Dict[int, np.ndarray] = {}
        self._gk_lapack: Dict[int, np.ndarray] = {}

    # ---- one-particle quantities (src/one_particle_quant_module.f90) ----
    def giw(self, n, i):
        return self.inp.giw[n + self.inp.iwmax, i]

    def _gmat_arg(self, n):
        """(i nu_n + mu - H(k) - dc - Sigma(nu_n)) for all k: (nkp, ndim, ndim)."""
        inp = self.inp
        g = -np.transpose(inp.hk, (2, 0, 1)).copy()
        d = np.arange(inp.ndim)
        g[:, d, d] = (CI * inp.iw_data[n + inp.iwmax] + inp.mu - inp.hk[d, d, :].T
                      - inp.dc[0, d] - inp.siw[n + inp.iwmax, d])
        return g

    def gk(self, n):
        """G(k, nu_n) for all k as built inside accumulate_chi0
        (src/one_particle_quant_module.f90:240-271): closed form for ndim<=3."""
        if n not in self._gk_cache:
            g = self._gmat_arg(n)
            nd = self.inp.ndim
            if nd == 1:
                g = 1.0 / g
            elif nd == 2:
                g = inverse_matrix_2(g)
            elif nd == 3:
                g = inverse_matrix_3(g)
            else:
                g = np.stack([inverse_matrix(x)[0] for x in g])
            self._gk_cache[n] = g
        return self._gk_cache[n]

    def gk_lapack(self, n):
        """G(k, nu_n) as get_gkiw builds it (src/one_particle_quant_module.f90:81-104):
        always a LAPACK inverse (batched here through numpy's LAPACK)."""
        if n not in self._gk_lapack:
            self._gk_lapack[n] = np.linalg.inv(self._gmat_arg(n))
        return self._gk_lapack[n]

    def get_chi0_loc(self, iwf, iwb):
        """Diagonal of chi0_loc({j,i}) = -beta g_i(nu) g_j(nu-omega) (:192-207)."""
        nd = self.inp.ndim
        out = np.empty(nd * nd, dtype=complex)
        for i in range(nd):
            for j in range(nd):
                out[i * nd + j] = -self.inp.beta * self.giw(iwf, i) * self.giw(iwf - iwb, j)
        return out

    def get_chi0_loc_inv(self, iwf, iwb):
        """Diagonal of chi0_loc^{-1} (:210-225)."""
        nd = self.inp.ndim
        out = np.empty(nd * nd, dtype=complex)
        for i in range(nd):
            for j in range(nd):
                out[i * nd + j] = -1.0 / (self.inp.beta * self.giw(iwf, i) * self.giw(iwf - iwb, j))
        return out

    def chi0_q(self, iq, iwf, iwb):
        """k-summed bubble of main.F90:649-654: sum_k accumulate_chi0 / nkp.

        chi0({i,j},{l,k}) = -(beta/nkp) sum_k G_il(k, nu) G_kj(k-q, nu-omega)
        (src/one_particle_quant_module.f90:274-288)."""
        inp = self.inp
        g1 = self.gk(iwf)
        g2 = self.gk(iwf - iwb)[self.kq_ind[:, iq] - 1]
        c = -inp.beta * np.einsum("nil,nkj->ijlk", g1, g2)
        return (c.reshape(inp.ndim2, inp.ndim2) / float(inp.nkp)).copy(order="F")

    # ---- susceptibility sums (src/susc_module.f90:34-56) ----
    def calc_chi_qw(self, chi_qw, interm3, chi0_sum):
        inp = self.inp
        nd2 = inp.ndim2
        tmp = np.zeros((nd2, nd2), dtype=complex)
        for dum in range(2 * inp.iwfmax_small):
            tmp += interm3[:, dum * nd2:(dum + 1) * nd2] @ chi0_sum[:, :, dum]
        chi_qw += tmp / inp.beta ** 2

    # ---- EOM (src/eom_module.f90) ----
    def n_fock(self):
        """get_nfock (src/one_particle_quant_module.f90:316-342): n(k, i, j) =
        2/beta sum_{nu>=0} Re G_DMFT(k, nu) + 1/2 on the diagonal."""
        if getattr(self, "_n_fock", None) is None:
            inp = self.inp
            acc = np.zeros((inp.nkp, inp.ndim, inp.ndim))
            for n in range(inp.iwmax):
                acc += self.gk_lapack(n).real
            nf = (2.0 * acc / inp.beta).astype(complex)
            for i in range(inp.ndim):
                nf[:, i, i] += 0.5
            self._n_fock = nf
        return self._n_fock

    def calc_eom_static(self, iq, sigma_dmft, sigma_hf=None):
        """calc_eom_static (src/eom_module.f90:39-111): local Hartree term into
        sigma_dmft for iq = 0; with V(q) the non-local Hartree 2 v(q=0) n_dmft
        (iq = 0) and the Fock term -v(q)/nqp n_fock(k-q) into sigma_hf."""
        inp = self.inp
        nd = inp.ndim
        if inp.vq is not None and sigma_hf is not None:
            v = inp.vq[:, :, iq]
            if iq == 0:
                for i in range(nd):
                    for j in range(nd):
                        sigma_hf[i, i, :] += 2.0 * v[i * nd + i, j * nd + j] * inp.n_dmft[j]
            nf = self.n_fock()
            ikq = self.kq_ind[:, iq] - 1
            for l in range(nd):
                for j in range(nd):
                    for i in range(nd):
                        for k in range(nd):
                            alpha = v[i * nd + k, l * nd + j] / inp.nqp
                            sigma_hf[i, l, :] -= alpha * nf[ikq, j, k]
        if iq == 0:
            tmp = np.zeros(nd, dtype=complex)
            for i in range(nd):
                i1 = i * nd + i
                for j in range(nd):
                    i2 = j * nd + j
                    i3 = i * nd + j
                    tmp[i] += (2.0 * inp.u[i1, i2] - inp.u[i3, i3]) * inp.n_dmft[j]
            for i in range(nd):
                sigma_dmft[i, i, :] += tmp[i]

    def calc_eom_dmft(self, gammawd, iwb, sigma_dmft):
        """Local Sigma from -U/beta * gamma^w_d (src/eom_module.f90:115-161)."""
        inp = self.inp
        nd, nd2, iwfs = inp.ndim, inp.ndim2, inp.iwfmax_small
        m_tot = (-1.0 / inp.beta) * (inp.u @ gammawd)
        for iwf in range(iwfs):
            for l in range(nd):
                for k in range(nd):
                    i2 = nd2 * (iwf + iwfs) + l * nd + k
                    for i in range(nd):
                        i1 = i * nd + k
                        sigma_dmft[i, l, iwf + iwfs] += m_tot[i1, i2] * self.giw(iwf - iwb, k)
            sigma_dmft[:, :, -iwf - 1 + iwfs] = np.conj(sigma_dmft[:, :, iwf + iwfs]).T

    def eom_m_tot(self, etaqd, etaqm, gammaqd, iq=None, gammawd=None):
        """m_tot of calc_eom_dynamic (src/eom_module.f90:184-207)."""
        inp = self.inp
        nqp = float(inp.nqp)
        v = inp.vq[:, :, iq] if inp.vq is not None else 0.0
        u_work = v + inp.u - 0.5 * inp.u_tilde
        m = (-1.0 / inp.beta / nqp) * (u_work @ etaqd)
        m += (1.5 / inp.beta / nqp) * (inp.u_tilde @ etaqm)
        m += (1.0 / inp.beta / nqp) * (inp.u @ gammaqd)
        if inp.vq is not None:
            m += (-1.0 / inp.beta / nqp) * (v @ gammawd)
        return m

    def calc_eom_dynamic(self, etaqd, etaqm, gammaqd, iwb, iq, sigma_nl, gammawd=None):
        """Sigma(i,l,nu,k) += m_tot({j,i},{k',l,nu}) G_jk'(k-q, nu-omega) for
        nu >= 0, then the mirror Sigma(-nu-1) = Sigma(nu)^dagger
        (src/eom_module.f90:165-233)."""
        inp = self.inp
        nd, nd2, iwfs = inp.ndim, inp.ndim2, inp.iwfmax_small
        m_tot = self.eom_m_tot(etaqd, etaqm, gammaqd, iq, gammawd)
        M = m_tot[:, nd2 * iwfs:].reshape(nd, nd, iwfs, nd, nd)   # [i, j, w, l, k']
        ikq = self.kq_ind[:, iq] - 1
        G = np.stack([self.gk_lapack(iwf - iwb)[ikq] for iwf in range(iwfs)], axis=1)  # [n, w, j, k']
        sig = np.einsum("ijwlk,nwjk->ilwn", M, G)
        sigma_nl[:, :, iwfs:, :] += sig
        for iwf in range(iwfs):
            sigma_nl[:, :, -iwf - 1 + iwfs, :] = np.conj(
                np.transpose(sigma_nl[:, :, iwf + iwfs, :], (1, 0, 2)))

    # ---- the (q, omega) loop: src/main.F90:484-799 ----
    def run(self, qw_points: Optional[Sequence[Tuple[int, int]]] = None):
        """Run the ladder loop over (iwb, iq) points (iq 0-based).

        Defaults to the full list with omega outer, q inner (main.F90:381-389).
        Returns the raw accumulators of the reference, keyed by its variable
        names, plus per-point BSE intermediates for the first point.
        """
        inp = self.inp
        nd, nd2, N, iwfs, iwbs = inp.ndim, inp.ndim2, inp.maxdim, inp.iwfmax_small, inp.iwbmax_small
        beta = inp.beta
        nw = 2 * iwbs + 1
        nqp = inp.nqp
        iwstart, iwstop = inp.iw_range
        if qw_points is None:
            qw_points = [(iwb, iq) for iwb in range(-iwbs, iwbs + 1) for iq in range(nqp)]
        npts = len(qw_points)
        out = dict(
            chi_qw_dens=np.zeros((nd2, nd2, npts), complex, order="F"),
            chi_qw_magn=np.zeros((nd2, nd2, npts), complex, order="F"),
            bubble_nl=np.zeros((nd2, nd2, npts), complex, order="F"),
            bubble_loc=np.zeros((nd2, nd2, nw), complex, order="F"),
            chi_loc_dens=np.zeros((nd2, nd2, nw), complex, order="F"),
            chi_loc_magn=np.zeros((nd2, nd2, nw), complex, order="F"),
            sigma_nl=np.zeros((nd, nd, 2 * iwfs, inp.nkp), complex, order="F"),
            sigma_dmft=np.zeros((nd, nd, 2 * iwfs), complex, order="F"),
            sigma_hf=np.zeros((nd, nd, inp.nkp), complex, order="F"),
            qw=np.array(qw_points, dtype=np.int64),
            status=np.zeros(npts, dtype=np.int32),
        )
        cur_iwb = None
        for p, (iwb, iq) in enumerate(qw_points):
            if iwb != cur_iwb:
                cur_iwb = iwb
                loc = self.local_block(iwb, iq, out)
            chi0w_inv, chi0w, bubble_loc_tmp, Fd, Fm, gd, gm, opgd, opgm = loc
            if inp.do_eom and iwb == 0 and (iq == 0 or inp.vq is not None):
                self.calc_eom_static(iq, out["sigma_dmft"], out["sigma_hf"])
            if inp.do_eom and iq == 0:
                self.calc_eom_dmft(gd, iwb, out["sigma_dmft"])
            res = self.point(iq, iwb, loc)
            if inp.do_chi:
                out["bubble_nl"][:, :, p] = res["bubble_nl"]
                out["chi_qw_dens"][:, :, p] = res["chi_qw_dens"]
                out["chi_qw_magn"][:, :, p] = res["chi_qw_magn"]
            if inp.do_eom:
                self.calc_eom_dynamic(res["etaqd"], res["etaqm"], res["gammaqd"], iwb, iq,
                                      out["sigma_nl"], gd)
            out["status"][p] = res["ierr"]
            if p == 0:
                out["first_point"] = res
        return out

    def local_block(self, iwb, iq, out):
        """Per-omega local quantities, main.F90:506-627."""
        inp = self.inp
        nd2, N, iwfs, beta = inp.ndim2, inp.maxdim, inp.iwfmax_small, inp.beta
        iwbs = inp.iwbmax_small
        iwstart, iwstop = inp.iw_range
        chi0w_inv = np.zeros((nd2, 2 * iwfs), complex, order="F")   # diagonals
        for iwf in range(-iwfs, iwfs):
            chi0w_inv[:, iwf + iwfs] = self.get_chi0_loc_inv(iwf, iwb)
        chi0w = np.zeros((nd2, nd2, 2 * iwfs), complex, order="F")
        bubble_loc_tmp = np.zeros((nd2, nd2), complex, order="F")
        if inp.do_chi:
            for iwf in range(iwstart, iwstop + 1):
                c = np.diag(self.get_chi0_loc(iwf, iwb))
                bubble_loc_tmp += c
                if -iwfs <= iwf <= iwfs - 1:
                    chi0w[:, :, iwf + iwfs] = c
            bubble_loc_tmp = bubble_loc_tmp / beta ** 2
            if iq == 0:
                out["bubble_loc"][:, :, iwb + iwbs] += bubble_loc_tmp
        chi_d, chi_m = inp.vertex(iwb)
        Fd = np.array(chi_d, dtype=complex, order="F")
        Fm = np.array(chi_m, dtype=complex, order="F")
        # transpose symmetrisation (main.F90:529-537)
        Fd = np.asfortranarray(0.5 * (Fd + Fd.T))
        Fm = np.asfortranarray(0.5 * (Fm + Fm.T))
        # F~ = chi_loc * chi0_loc^-1 - 1 (main.F90:542-553)
        scale = chi0w_inv.T.reshape(-1)         # index i = i2 + dum*nd2
        Fd *= scale[None, :]
        Fm *= scale[None, :]
        Fd[np.arange(N), np.arange(N)] -= 1.0
        Fm[np.arange(N), np.arange(N)] -= 1.0
        # gamma^w (main.F90:559-571): external three-leg vertex or the F~ row sums
        if inp.threeleg is not None:
            gd, gm = (np.array(x, dtype=complex, order="F") for x in inp.threeleg(iwb))
        else:
            gd = np.zeros((nd2, N), complex, order="F")
            gm = np.zeros((nd2, N), complex, order="F")
            for dum in range(2 * iwfs):
                gd += Fd[dum * nd2:(dum + 1) * nd2, :]
                gm += Fm[dum * nd2:(dum + 1) * nd2, :]
        if iq == 0 and inp.do_chi and inp.chi_loc_ext is None:
            self.calc_chi_qw(out["chi_loc_dens"][:, :, iwb + iwbs], gd, chi0w)
            self.calc_chi_qw(out["chi_loc_magn"][:, :, iwb + iwbs], gm, chi0w)
        opgd = gd.copy(order="F")
        opgm = gm.copy(order="F")
        for i1 in range(nd2):
            for dum in range(2 * iwfs):
                opgd[i1, i1 + dum * nd2] += 1.0
                opgm[i1, i1 + dum * nd2] += 1.0
        return chi0w_inv, chi0w, bubble_loc_tmp, Fd, Fm, gd, gm, opgd, opgm

    def point(self, iq, iwb, loc):
        """Non-local part of one (q, omega) point, main.F90:644-781 (no EOM accumulation)."""
        inp = self.inp
        nd2, N, iwfs, beta = inp.ndim2, inp.maxdim, inp.iwfmax_small, inp.beta
        chi0w_inv, chi0w, bubble_loc_tmp, Fd, Fm, gd, gm, opgd, opgm = loc
        iwstart, iwstop = inp.iw_range
        chi0q = np.zeros((nd2, nd2, 2 * iwfs), complex, order="F")
        bub = np.zeros((nd2, nd2), complex, order="F")
        for iwf in range(iwstart, iwstop + 1):
            c = self.chi0_q(iq, iwf, iwb)
            bub += c
            if -iwfs <= iwf <= iwfs - 1:
                chi0q[:, :, iwf + iwfs] = c
        res = {"chi0q": chi0q}
        if inp.do_chi:
            res["bubble_nl"] = bub / beta ** 2 - bubble_loc_tmp
            chi0nl = chi0q - chi0w
            cd = np.zeros((nd2, nd2), complex, order="F")
            cm = np.zeros((nd2, nd2), complex, order="F")
            self.calc_chi_qw(cd, gd, chi0nl)
            self.calc_chi_qw(cm, gm, chi0nl)
        # BSE build (main.F90:674-732)
        bd = np.zeros((N, N), complex, order="F")
        bm = np.zeros((N, N), complex, order="F")
        gammaqd = np.zeros((nd2, N), complex, order="F")
        for dum1 in range(2 * iwfs):
            off = dum1 * nd2
            sw = chi0q[:, :, dum1] * chi0w_inv[None, :, dum1]
            sw[np.arange(nd2), np.arange(nd2)] -= 1.0
            rect = sw @ Fd[off:off + nd2, :]
            bd[off:off + nd2, :] = -rect
            gammaqd += rect
            rect = sw @ Fm[off:off + nd2, :]
            bm[off:off + nd2, :] = -rect
            if inp.vq is not None:     # density channel: 2 beta^-2 chi0^q v^q (1+gamma^w_d) (:710-719)
                small = (2.0 / beta ** 2) * (chi0q[:, :, dum1] @ inp.vq[:, :, iq])
                bd[off:off + nd2, :] -= small @ opgd
        bd[np.arange(N), np.arange(N)] += 1.0
        bm[np.arange(N), np.arange(N)] += 1.0
        res["A_dens"] = bd.copy(order="F")
        res["A_magn"] = bm.copy(order="F")
        # inversion (main.F90:734-737)
        invd, erd, _ = inverse_matrix(bd)
        invm, erm, _ = inverse_matrix(bm)
        res["ierr"] = erd if erd != 0 else erm
        invd[np.arange(N), np.arange(N)] -= 1.0
        invm[np.arange(N), np.arange(N)] -= 1.0
        etaqd = opgd @ invd
        etaqm = opgm @ invm
        res.update(etaqd=etaqd, etaqm=etaqm, gammaqd=gammaqd)
        if inp.do_chi:
            self.calc_chi_qw(cd, etaqd, chi0q)
            self.calc_chi_qw(cm, etaqm, chi0q)
            res["chi_qw_dens"] = cd
            res["chi_qw_magn"] = cm
        return res


def assemble(inp: LadderInputs, out):
    """Post-loop assembly: chi_loc += bubble_loc (main.F90:935-936);
    chi(q,w) = chi_nl + bubble_nl + chi_loc(w) (main.F90:1050,1059-1063,1127,1136-1140);
    Sigma = Sigma_nl + siw on the diagonal (add_siw_dmft, src/eom_module.f90:237-251)."""
    iwbs, iwfs, nd = inp.iwbmax_small, inp.iwfmax_small, inp.ndim
    if inp.chi_loc_ext is not None:   # read from file: already contains the bubble (main.F90:933-936)
        chi_loc_d = np.asarray(inp.chi_loc_ext[0])
        chi_loc_m = np.asarray(inp.chi_loc_ext[1])
    else:
        chi_loc_d = out["chi_loc_dens"] + out["bubble_loc"]
        chi_loc_m = out["chi_loc_magn"] + out["bubble_loc"]
    qw = out["qw"]
    widx = qw[:, 0] + iwbs
    chi_d = out["chi_qw_dens"] + out["bubble_nl"] + chi_loc_d[:, :, widx]
    chi_m = out["chi_qw_magn"] + out["bubble_nl"] + chi_loc_m[:, :, widx]
    sig = out["sigma_nl"].copy(order="F")
    for b in range(nd):
        sig[b, b, :, :] += inp.siw[np.arange(-iwfs, iwfs) + inp.iwmax, b][:, None]
    return dict(chi_dens=chi_d, chi_magn=chi_m, chi_loc_dens=chi_loc_d,
                chi_loc_magn=chi_loc_m, sigma=sig)


def _gkiw_dga(inp: LadderInputs, ik, n, skiw):
    """get_gkiw_dga (src/one_particle_quant_module.f90:106-126): lattice G at k-point
    ik (0-based, full mesh), Matsubara n, with any self-energy skiw (ndim x ndim)."""
    nd = inp.ndim
    g = -inp.hk[:, :, ik] - skiw
    for i in range(nd):
        g[i, i] = 1j * inp.iw_data[n + inp.iwmax] + inp.mu - inp.hk[i, i, ik] - inp.dc[0, i] - skiw[i, i]
    return inverse_matrix(g)[0]


def post_loop(inp: LadderInputs, sigma_sum, k_data_eom=None):
    """src/main.F90:869-890 on the reduced non-local self-energy
    sigma_sum(ndim, ndim, 2*iwf, nkp_eom):
      add_siw_dmft    (src/eom_module.f90:237-251),
      get_sigma_g_loc (src/one_particle_quant_module.f90:129-187; full k mesh only),
      get_ndga        (src/one_particle_quant_module.f90:344-394).
    k_data_eom: 1-based full-mesh k indices of the EOM k-points (None = full mesh)."""
    nd, iwf, iwmax, beta = inp.ndim, inp.iwfmax_small, inp.iwmax, inp.beta
    sig = np.array(sigma_sum, dtype=complex, order="F")
    nk_eom = sig.shape[3]
    for ik in range(nk_eom):                       # add_siw_dmft
        for w in range(-iwf, iwf):
            for b in range(nd):
                sig[b, b, w + iwf, ik] += inp.siw[w + iwmax, b]
    out = {"sigma_sum": sig}
    diag_siw = lambda n: np.diag(inp.siw[n + iwmax, :])
    if k_data_eom is None and nk_eom == inp.nkp:   # get_sigma_g_loc
        nkp = inp.nkp
        sloc = sig.sum(axis=3) / nkp
        gloc = np.zeros((2 * iwmax, nd, nd), complex)
        for ik in range(nkp):
            for n in range(0, iwf):
                gloc[n + iwmax] += _gkiw_dga(inp, ik, n, sig[:, :, n + iwf, ik])
            for n in range(iwf, iwmax):
                gloc[n + iwmax] += _gkiw_dga(inp, ik, n, diag_siw(n))
        for n in range(0, iwmax):
            gloc[-n - 1 + iwmax] = gloc[n + iwmax].conj().T
        out["sigma_loc"] = np.asfortranarray(sloc)
        out["gloc"] = np.asfortranarray(gloc / nkp)
    kmap = (np.arange(nk_eom) if k_data_eom is None else np.asarray(k_data_eom) - 1)
    nk = np.zeros((nk_eom, nd, nd), complex)
    for ik in range(nk_eom):                       # get_ndga
        for n in range(0, iwf):
            nk[ik] += _gkiw_dga(inp, kmap[ik], n, sig[:, :, n + iwf, ik]).real
        for n in range(iwf, iwmax):
            nk[ik] += _gkiw_dga(inp, kmap[ik], n, diag_siw(n)).real
        nk[ik] = 2.0 * nk[ik] / beta
        for i in range(nd):
            nk[ik, i, i] += 0.5
    out["n_dga_k"] = np.asfortranarray(nk)
    out["n_dga"] = np.array([nk[:, i, i].sum() for i in range(nd)]) / nk_eom
    return out


def read_threeleg_transform(g3_dens, g3_magn, iwb, ndims, giw, n_dmft, beta, iwf, iwmax):
    """The transform part of read_threeleg (src/hdf5_module.f90:820-880): the
    three-leg vertex g3(ndim, ndim, ndim, ndim, 2*n3iwf) as w2dynamics stores it
    (index m + n3iwf holds Matsubara m, before the beta factor of :829,838) ->
    gamma^w(ndim2, maxdim) with the disconnected parts and the division by
    -G G in the correlated subspace."""
    nd = g3_dens.shape[0]
    n3iwf = g3_dens.shape[4] // 2
    nd2 = nd * nd
    gtd = np.asarray(g3_dens) * beta
    gtm = np.asarray(g3_magn) * beta
    gd = np.zeros((nd2, nd2 * 2 * iwf), complex)
    gm = np.zeros((nd2, nd2 * 2 * iwf), complex)
    g = lambda n, b: giw[n + iwmax, b]
    i1 = 0
    for i in range(nd):
        for j in range(nd):
            i2 = 0
            for w in range(2 * iwf):
                nu = w - iwf
                for k in range(nd):
                    for l in range(nd):
                        c4 = _index2cor(ndims, i + 1, j + 1, k + 1, l + 1)
                        vd = gtd[k, l, j, i, n3iwf + w - iwf]
                        vm = gtm[k, l, j, i, n3iwf + w - iwf]
                        if i == j and k == l and iwb == 0 and c4:
                            vd = vd + 2.0 * beta * (1.0 - n_dmft[i]) * g(nu, k)
                        if i == k and j == l and c4:
                            t = g(nu, k) * g(nu - iwb, l)
                            vd = vd + t
                            vm = vm + t
                        if c4:
                            den = -1.0 * g(nu, k) * g(nu - iwb, l)
                            vd = vd / den
                            vm = vm / den
                        gd[i1, i2] = vd
                        gm[i1, i2] = vm
                        i2 += 1
            i1 += 1
    return np.asfortranarray(gd), np.asfortranarray(gm)


def read_chi_loc_transform(chi_raw, channel, ndims, giw, n_dmft, beta, iwbs, iwmax):
    """The transform part of read_chi_loc (src/hdf5_module.f90:958-993): the
    frequency-summed local susceptibility chi(ndim, ndim, ndim, ndim, 2*n2iwb+1)
    as w2dynamics stores it (index m + n2iwb holds bosonic m) -> chi_loc(ndim2,
    ndim2, -iwbs:iwbs) with the dens-channel omega = 0 term and, when the model
    has more than one impurity or uncorrelated bands, the lattice bubble of the
    uncorrelated legs."""
    nd = chi_raw.shape[0]
    n2iwb = chi_raw.shape[4] // 2
    nd2 = nd * nd
    extend = not (len(ndims) >= 1 and ndims[0][0] == nd)
    sl = np.asarray(chi_raw)[..., n2iwb - iwbs:n2iwb + iwbs + 1]
    out = np.zeros((nd2, nd2, 2 * iwbs + 1), complex)
    g = lambda n, b: giw[n + iwmax, b]
    i1 = 0
    for i in range(nd):
        for j in range(nd):
            i2 = 0
            for k in range(nd):
                for l in range(nd):
                    out[i1, i2, :] = sl[i, j, l, k, :]
                    c4 = _index2cor(ndims, i + 1, j + 1, k + 1, l + 1)
                    if c4 and i == j and k == l and channel == "dens":
                        out[i1, i2, iwbs] -= 2.0 * beta * (1.0 - n_dmft[i]) * (1.0 - n_dmft[k])
                    if extend and not c4 and i == k and j == l:
                        for w in range(-iwbs, iwbs + 1):
                            for n in range(-iwmax + iwbs, iwmax - iwbs):
                                out[i1, i2, w + iwbs] -= g(n, i) * g(n - w, j) / beta
                    i2 += 1
            i1 += 1
    return np.asfortranarray(out)


def read_vq_transform(vq_raw):
    """The index map of read_vq (src/interaction_module.f90:107-119):
    vq(i, j, k, l, q) -> v(i1 = i*ndim + k, i2 = l*ndim + j, q)."""
    vq_raw = np.asarray(vq_raw)
    nd, nqp = vq_raw.shape[0], vq_raw.shape[4]
    v = np.zeros((nd * nd, nd * nd, nqp), complex)
    for l in range(nd):
        for j in range(nd):
            for i in range(nd):
                for k in range(nd):
                    v[i * nd + k, l * nd + j, :] = vq_raw[i, j, k, l, :]
    return np.asfortranarray(v)
