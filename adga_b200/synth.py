"""Seeded synthetic inputs for the ladder hot path.

The reference reads H(k) from a ``.hk`` file, the DMFT self-energy and Green's
function from HDF5 and the local generalised susceptibility chi_loc(nu, nu';
omega) from the vertex file (``read_vertex``, src/hdf5_module.f90:629-773).
None of those files exist here, so this module builds inputs of the same
shapes and value ranges:

* H(k) on an nkx*nky*nkz grid, ordered kz-fastest like the ``.hk`` files
  (src/kq_tools.f90:119-144), coordinates in [0, 1);
* Sigma(i nu) = A / (i nu + i gamma sgn nu), a causal second-order-like local
  self-energy; mu fixed by the requested filling (bisection on the lattice
  occupation with the reference's +1/2 convention,
  src/one_particle_quant_module.f90:295-313);
* G_imp(i nu) = 1 / (i nu + mu - Delta(i nu) - Sigma(i nu)) with a
  semicircular hybridisation Delta of half-width D;
* chi_loc^ch(omega) = (chi0_loc^-1 + Gamma_ch)^-1 in the reference's compound
  layout (i1 + nu*ndim2, i2 + nu'*ndim2) with
  Gamma_ch = s_ch / beta^2 * kron(1 + eps * P, V_ch), V_d = 2u - u~,
  V_m = -u~ (s_ch = +1), P a seeded Hermitian nu<->nu' perturbation, eps = 1%.

Everything is FP64 / complex128 and deterministic in the seed.
"""
from __future__ import annotations

import dataclasses
import math
from dataclasses import dataclass, field
from functools import lru_cache
from typing import Dict, Optional, Tuple

import numpy as np


@dataclass
class Spec:
    name: str
    ndim: int
    nk: Tuple[int, int, int]
    nq: Tuple[int, int, int]
    iwf: int                 # iwfmax_small: 2*iwf fermionic frequencies
    iwb: int                 # iwbmax_small: 2*iwb+1 bosonic frequencies
    beta: float
    U: float
    J: float = 0.0
    V: Optional[float] = None    # inter-orbital; default U - 2J
    model: str = "sc"
    hop: Dict[str, float] = field(default_factory=dict)
    filling: float = 0.5         # per spin-orbital
    D: float = 1.0               # semicircular half-width of Delta
    sigma_gamma: float = 0.5     # damping of the synthetic self-energy
    sigma_A: float = 0.5         # Sigma(i nu) = sigma_A*U*n(1-n) / (i nu + i gamma sgn nu)
    vertex_eps: float = 0.01
    iwmax: Optional[int] = None
    seed: int = 1234
    offdiag: float = 0.0         # inter-orbital hopping amplitude (test models)

    @property
    def ndim2(self): return self.ndim * self.ndim
    @property
    def maxdim(self): return self.ndim2 * 2 * self.iwf
    @property
    def nkp(self): return self.nk[0] * self.nk[1] * self.nk[2]
    @property
    def nqp(self): return self.nq[0] * self.nq[1] * self.nq[2]
    @property
    def n_iwmax(self): return self.iwmax if self.iwmax else 4 * (self.iwf + self.iwb)
    @property
    def Vval(self): return self.U - 2 * self.J if self.V is None else self.V


# The five workloads of the benchmark suite (sizes, couplings, grids) and
# small models used by the parity tests.
SPECS: Dict[str, Spec] = {
    # single-orbital simple cubic, t = 0.25, 10^3 k / 5^3 q, U = 2, beta = 10, half filling
    "c0": Spec("c0", 1, (10, 10, 10), (5, 5, 5), 20, 10, 10.0, 2.0, model="sc",
               hop=dict(t=0.25), filling=0.5, seed=1234),
    # SrVO3-like t2g: t=0.26, t'=0.03, t''=0.08 on 20^3 k / 10^3 q, Kanamori U=5 J=0.75 V=3.5
    "c1": Spec("c1", 3, (20, 20, 20), (10, 10, 10), 60, 10, 10.0, 5.0, 0.75, 3.5, model="t2g",
               hop=dict(t=0.26, tp=0.03, tpp=0.08), filling=1.0 / 6.0, seed=1235),
    # two-orbital e_g: t=0.3, anisotropy 0.5, 16^3 k / 8^3 q, U=4 J=0.6, beta=20
    "c3": Spec("c3", 2, (16, 16, 16), (8, 8, 8), 40, 5, 20.0, 4.0, 0.6, model="eg",
               hop=dict(t=0.3, aniso=0.5), filling=0.25, seed=1237),
    # parity-test models (small; inter-orbital complex hopping exercises every index)
    "t1": Spec("t1", 1, (4, 4, 4), (2, 2, 2), 4, 2, 10.0, 2.0, model="sc",
               hop=dict(t=0.25), filling=0.4, seed=11),
    "t2": Spec("t2", 2, (4, 4, 2), (2, 2, 1), 3, 1, 8.0, 3.0, 0.5, model="eg",
               hop=dict(t=0.3, aniso=0.5), filling=0.3, seed=12, offdiag=0.05),
    "t3": Spec("t3", 3, (4, 2, 2), (2, 1, 1), 3, 1, 10.0, 4.0, 0.6, model="t2g",
               hop=dict(t=0.26, tp=0.03, tpp=0.08), filling=0.2, seed=13, offdiag=0.04),
    "t3b": Spec("t3b", 3, (6, 6, 6), (3, 3, 3), 8, 2, 10.0, 5.0, 0.75, 3.5, model="t2g",
                hop=dict(t=0.26, tp=0.03, tpp=0.08), filling=1.0 / 6.0, seed=14, offdiag=0.03),
    "t3m": Spec("t3m", 3, (4, 4, 4), (2, 2, 2), 12, 1, 10.0, 5.0, 0.75, 3.5, model="t2g",
                hop=dict(t=0.26, tp=0.03, tpp=0.08), filling=1.0 / 6.0, seed=16, offdiag=0.03),
    "t5": Spec("t5", 5, (2, 2, 2), (2, 1, 1), 2, 1, 10.0, 3.0, 0.5, model="d5",
               hop=dict(t=0.2, t2=0.12), filling=0.3, seed=15, offdiag=0.03),
}
SPECS["c2"] = Spec(**{**SPECS["c1"].__dict__, "name": "c2"})
# the differentiation model on a 4^3 k / 2^3 q sub-grid (dense-Jacobian checks): BSE 320 x 320
SPECS["c3s"] = Spec(**{**SPECS["c3"].__dict__, "name": "c3s", "nk": (4, 4, 4), "nq": (2, 2, 2)})


def sweep_specs(n=64, seed=4321):
    """The uneven-size parameter sweep: ndim in {1,3,5}, U in [2,6], J/U in
    [0.1,0.2], beta in {10,20,40}, iwf in {20,40,80}, 12^3 k / 6^3 q, 11 omega."""
    rng = np.random.default_rng(seed)
    out = []
    for p in range(n):
        nd = int(rng.choice([1, 3, 5]))
        U = float(rng.uniform(2, 6))
        J = 0.0 if nd == 1 else U * float(rng.uniform(0.1, 0.2))
        beta = float(rng.choice([10.0, 20.0, 40.0]))
        iwf = int(rng.choice([20, 40, 80]))
        hop = dict(t=float(rng.uniform(0.1, 0.35)), t2=float(rng.uniform(0.1, 0.35)))
        out.append(Spec(f"sweep{p}", nd, (12, 12, 12), (6, 6, 6), iwf, 5, beta, U, J,
                        model="sc" if nd == 1 else "d5", hop=hop, filling=0.4,
                        seed=seed + 17 * p))
    return out


# ----------------------------------------------------------------------------
def k_points(nk):
    """Fractional k coordinates in .hk order (kz fastest)."""
    nx, ny, nz = nk
    ix, iy, iz = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    return np.stack([ix.ravel() / nx, iy.ravel() / ny, iz.ravel() / nz], axis=0)


def hamiltonian(spec: Spec) -> np.ndarray:
    """H(k) as (ndim, ndim, nkp) complex, Fortran order."""
    kd = k_points(spec.nk) * 2 * np.pi
    cx, cy, cz = np.cos(kd)
    sx, sy, sz = np.sin(kd)
    nd, nkp = spec.ndim, spec.nkp
    H = np.zeros((nd, nd, nkp), dtype=complex, order="F")
    h = spec.hop
    if spec.model == "sc":
        eps = [-2 * h["t"] * (cx + cy + cz)] * nd
    elif spec.model == "t2g":
        t, tp, tpp = h["t"], h["tp"], h["tpp"]
        exy = -2 * t * (cx + cy) - 2 * tp * cz - 4 * tpp * cx * cy
        exz = -2 * t * (cx + cz) - 2 * tp * cy - 4 * tpp * cx * cz
        eyz = -2 * t * (cy + cz) - 2 * tp * cx - 4 * tpp * cy * cz
        eps = [exy, exz, eyz][:nd]
    elif spec.model == "eg":
        t, a = h["t"], h["aniso"]
        eps = [-2 * t * (cx + cy + a * cz), -2 * t * (a * cx + a * cy + cz)][:nd]
    elif spec.model == "d5":
        t, t2 = h["t"], h["t2"]
        base = -2 * t * (cx + cy + cz) - 4 * t2 * (cx * cy + cy * cz + cx * cz)
        eps = [base * (1.0 + 0.15 * a) + 0.05 * a for a in range(nd)]
    else:
        raise ValueError(spec.model)
    for a in range(nd):
        H[a, a, :] = eps[a]
    if spec.offdiag:
        # Hermitian inter-orbital terms with complex phases (test models only)
        for a in range(nd):
            for b in range(a + 1, nd):
                v = spec.offdiag * ((1 + 0.3 * a) * sx * sy + 0.7j * (b - a) * sz * cx + 0.2 * cz)
                H[a, b, :] = v
                H[b, a, :] = np.conj(v)
    return H


def kanamori_umat(nd, U, V, J):
    """U_ijkl for one impurity with only correlated bands (interaction_mode 1)."""
    Um = np.zeros((nd,) * 4)
    for i in range(nd):
        for j in range(nd):
            Um[i, i, j, j] = U if i == j else J
            if i != j:
                Um[i, j, i, j] = V
                Um[i, j, j, i] = J
    return Um


def compound_u(Um):
    """u({k,i},{j,l}) = U_ijkl, u~({k,i},{j,l}) = U_ijlk (i1 = i*nd+k, i2 = l*nd+j)."""
    nd = Um.shape[0]
    u = np.zeros((nd * nd, nd * nd), dtype=complex, order="F")
    ut = np.zeros_like(u)
    for l in range(nd):
        for j in range(nd):
            for i in range(nd):
                for k in range(nd):
                    u[i * nd + k, l * nd + j] = Um[i, j, k, l]
                    ut[i * nd + k, l * nd + j] = Um[i, j, l, k]
    return u, ut


@dataclass
class Problem:
    spec: Spec
    iwmax: int
    beta: float
    mu: float
    iw_data: np.ndarray
    hk: np.ndarray
    siw: np.ndarray
    giw: np.ndarray
    dc: np.ndarray
    u: np.ndarray
    u_tilde: np.ndarray
    n_dmft: np.ndarray
    Umat: np.ndarray
    _vcache: Dict[int, Tuple[np.ndarray, np.ndarray]] = field(default_factory=dict, repr=False)

    @property
    def ndim(self): return self.spec.ndim
    @property
    def ndim2(self): return self.spec.ndim2
    @property
    def maxdim(self): return self.spec.maxdim
    @property
    def nkp(self): return self.spec.nkp
    @property
    def nqp(self): return self.spec.nqp

    def vertex(self, iwb: int):
        """(chi_loc_dens, chi_loc_magn) at bosonic index iwb: (maxdim, maxdim), F-order."""
        if iwb not in self._vcache:
            self._vcache[iwb] = _make_vertex(self, iwb)
        return self._vcache[iwb]

    def clear_vertex_cache(self):
        self._vcache.clear()


def _sigma(spec: Spec, iw: np.ndarray):
    nd = spec.ndim
    n = spec.filling
    A = spec.sigma_A * spec.U * n * (1 - n)
    s = A / (1j * iw + 1j * spec.sigma_gamma * np.sign(iw))
    return np.repeat(s[:, None], nd, axis=1)


def _lattice_filling(spec, H, iw_pos, sig_pos, mu, beta):
    """Per-orbital occupation with the +1/2 convention of get_ndmft/get_nfock.

    The synthetic self-energy is the same on every orbital, so
    G_aa(k, nu) = sum_b |V_ab(k)|^2 / (i nu + mu - E_b(k) - Sigma(nu)) with
    H(k) = V E V^dagger."""
    E, V = np.linalg.eigh(np.transpose(H, (2, 0, 1)))          # (nk, nd), (nk, nd, nd)
    w = np.abs(V) ** 2                                          # [k, a, b]
    g = 1.0 / (1j * iw_pos[None, None, :] + mu - E[:, :, None] - sig_pos[None, None, :, 0])
    f = 2.0 * np.real(g).sum(axis=2) / beta + 0.5               # [k, b]
    return np.einsum("kab,kb->a", w, f) / H.shape[2]


def make_problem(spec_or_name, quick_mu: bool = False) -> Problem:
    spec = SPECS[spec_or_name] if isinstance(spec_or_name, str) else spec_or_name
    beta = spec.beta
    iwmax = spec.n_iwmax
    nvals = np.arange(-iwmax, iwmax)
    iw = np.pi * (2 * nvals + 1) / beta
    H = hamiltonian(spec)
    siw = np.asfortranarray(_sigma(spec, iw))
    # chemical potential
    if abs(spec.filling - 0.5) < 1e-12 and spec.model == "sc" and not spec.offdiag:
        mu = 0.0
    else:
        sub = H
        ipos = iw[iwmax:]
        spos = siw[iwmax:]
        lo, hi = -12.0, 12.0
        for _ in range(48 if not quick_mu else 20):
            mid = 0.5 * (lo + hi)
            nn = _lattice_filling(spec, sub, ipos, spos, mid, beta).mean()
            if nn > spec.filling:
                hi = mid
            else:
                lo = mid
        mu = 0.5 * (lo + hi)
    # impurity Green's function with a semicircular hybridisation
    D = spec.D
    delta = 0.5 * (1j * iw - 1j * np.sign(iw) * np.sqrt(iw ** 2 + D ** 2))
    giw = 1.0 / (1j * iw[:, None] + mu - delta[:, None] - siw)
    giw = np.asfortranarray(giw)
    n_dmft = 2 * np.real(giw[iwmax:].sum(axis=0)) / beta + 0.5
    Um = kanamori_umat(spec.ndim, spec.U, spec.Vval, spec.J)
    u, ut = compound_u(Um)
    dc = np.zeros((2, spec.ndim), dtype=complex, order="F")
    return Problem(spec=spec, iwmax=iwmax, beta=beta, mu=float(mu), iw_data=iw, hk=H,
                   siw=siw, giw=giw, dc=dc, u=u, u_tilde=ut, n_dmft=n_dmft.astype(complex),
                   Umat=Um)


def chi0_loc_diag(prob: Problem, iwb: int) -> np.ndarray:
    """Diagonal of chi0_loc in the big compound index (i2 + dum*ndim2)."""
    nd, iwf, beta, iwmax = prob.ndim, prob.spec.iwf, prob.beta, prob.iwmax
    out = np.empty(prob.maxdim, dtype=complex)
    for dum in range(2 * iwf):
        n = dum - iwf
        for i in range(nd):
            for j in range(nd):
                out[dum * nd * nd + i * nd + j] = (-beta * prob.giw[n + iwmax, i]
                                                    * prob.giw[n - iwb + iwmax, j])
    return out


def _make_vertex(prob: Problem, iwb: int):
    spec = prob.spec
    n2 = 2 * spec.iwf
    c0 = chi0_loc_diag(prob, iwb)
    out = []
    for ch, (sgn, V) in enumerate(((1.0, 2 * prob.u - prob.u_tilde), (1.0, -prob.u_tilde))):
        rng = np.random.default_rng([spec.seed, iwb + 1000, ch])
        R = rng.uniform(-1, 1, (n2, n2)) + 1j * rng.uniform(-1, 1, (n2, n2))
        P = 0.5 * (R + R.conj().T)
        W = 1.0 + spec.vertex_eps * P
        Gam = (sgn / prob.beta ** 2) * np.kron(W, V)
        M = np.diag(1.0 / c0) + Gam
        out.append(np.asfortranarray(np.linalg.inv(M)))
    return out[0], out[1]


# ---------------------------------------------------------------------------
# Parameter derivatives of the synthetic model (inputs of the tangent ladder)
# ---------------------------------------------------------------------------
PARAMS = ("U", "J", "t")


def _vertex_parts(prob: Problem, iwb: int):
    """(W_d, V_d), (W_m, V_m) of _make_vertex: Gamma_ch = kron(W_ch, V_ch) / beta^2."""
    spec = prob.spec
    n2 = 2 * spec.iwf
    parts = []
    for ch, V in enumerate((2 * prob.u - prob.u_tilde, -prob.u_tilde)):
        rng = np.random.default_rng([spec.seed, iwb + 1000, ch])
        R = rng.uniform(-1, 1, (n2, n2)) + 1j * rng.uniform(-1, 1, (n2, n2))
        P = 0.5 * (R + R.conj().T)
        parts.append((1.0 + spec.vertex_eps * P, V))
    return parts


def tangent_inputs(prob: Problem, param: str):
    """Input tangents (dhk, du, du_tilde, dvertex(iwb)) of the ladder for one
    model parameter at fixed DMFT one-particle inputs (siw, giw, mu, n_dmft):
      U, J  Kanamori tensors with V = U - 2J (linear: du = u at unit couplings),
            and the local vertex chi_loc = (chi0_loc^-1 + Gamma(u, u~))^-1:
            dchi_loc = -chi_loc dGamma chi_loc;
      t     the hopping scale: dH/dt (H is linear in t)."""
    spec = prob.spec
    nd = spec.ndim
    if param == "t":
        hop = dict(spec.hop)
        hop["t"] = hop["t"] + 1.0
        dhk = hamiltonian(dataclasses.replace(spec, hop=hop)) - hamiltonian(spec)
        return np.asfortranarray(dhk), None, None, None
    if param not in ("U", "J"):
        raise ValueError(param)
    cU, cV, cJ = (1.0, 1.0, 0.0) if param == "U" else (0.0, -2.0, 1.0)
    du, dut = compound_u(kanamori_umat(nd, cU, cV, cJ))

    def dvertex(iwb):
        chis = prob.vertex(iwb)
        out = []
        for (W, _), chi, dV in zip(_vertex_parts(prob, iwb), chis, (2 * du - dut, -dut)):
            dG = np.kron(W, dV) / prob.beta ** 2
            out.append(np.asfortranarray(-chi @ dG @ chi))
        return out[0], out[1]

    return None, du, dut, dvertex


def perturbed_problem(prob: Problem, dU=0.0, dJ=0.0, dt=0.0) -> Problem:
    """The same problem with U, J (V = U - 2J) and the hopping scale t moved,
    the DMFT one-particle inputs (siw, giw, mu, n_dmft) kept: finite-difference
    checks of the tangent ladder."""
    spec = prob.spec
    hop = dict(spec.hop)
    if dt:
        hop["t"] = hop["t"] + dt
    V = (spec.Vval + dU - 2 * dJ)
    s2 = dataclasses.replace(spec, U=spec.U + dU, J=spec.J + dJ, V=V, hop=hop)
    Um = kanamori_umat(s2.ndim, s2.U, s2.Vval, s2.J)
    u, ut = compound_u(Um)
    return dataclasses.replace(prob, spec=s2, hk=hamiltonian(s2), u=u, u_tilde=ut, Umat=Um, _vcache={})
