"""CPU checks of two algorithmic choices of the GPU path against the oracle's
own data (numpy restatements, no GPU):

* the bubble and the EOM are cyclic correlations / convolutions over the k
  mesh, so they equal DFT products, and sampling the inverse transform on the
  q sub-mesh equals folding the products onto it (the transform path of
  k_dft.cu);
* the transposed BSE matrices 1 - D F~ factor without row interchanges with
  growth factor ~1, and that unpivoted FP32 LU contracts FP64 iterative
  refinement as fast as a pivoted one (the mixed path's factorisation).
"""
import numpy as np
import scipy.linalg as sl

from oracle import adga_oracle as O
from tests.helpers import problem, to_inputs


def kgrid_coords(nk, k):
    return k // (nk[1] * nk[2]), (k // nk[2]) % nk[1], k % nk[2]


def test_bubble_is_a_dft_product_and_folds_onto_the_q_mesh():
    p = problem("t3b")
    s = p.spec
    inp = to_inputs(p)
    orc = O.Oracle(inp)
    nd, nk, nkp = s.ndim, s.nk, int(np.prod(s.nk))
    qs = O.generate_q_vol(nk, s.nq) - 1
    for iwf, iwb in ((0, 0), (-3, 1), (2, -2)):
        A = orc.gk(iwf).reshape(*nk, nd, nd)               # G_il(k, nu)
        B = orc.gk(iwf - iwb).reshape(*nk, nd, nd)         # G_k'j(k, nu - omega)
        Ah = np.fft.fftn(A, axes=(0, 1, 2))
        Bh = np.fft.fftn(B, axes=(0, 1, 2))
        Bm = np.roll(np.flip(Bh, axis=(0, 1, 2)), 1, axis=(0, 1, 2))    # B^(-p)
        # corr[q](i, l, k', j) = sum_k A_il(k) B_k'j(k - q) = ifft(A^(p) B^(-p))
        corr = np.fft.ifftn(np.einsum("xyzil,xyzkj->xyzilkj", Ah, Bm), axes=(0, 1, 2))
        m = tuple(n // q for n, q in zip(nk, s.nq))
        for iq, qk in enumerate(qs):
            want = orc.chi0_q(iq, iwf, iwb)                # chi0({i,j},{l,k'}), i1 = i nd + j, i2 = l nd + k'
            c = corr[kgrid_coords(nk, qk)] * (-p.beta / nkp)
            got = np.einsum("ilkj->ijlk", c).reshape(nd * nd, nd * nd)
            assert np.max(np.abs(got - want)) < 1e-12 * np.max(np.abs(want))
        # folding the products onto the q mesh (q = m a) and transforming there samples the same values
        prod = Ah[..., 0, 0] * Bm[..., 0, 0]
        mesh = np.zeros(s.nq, dtype=complex)
        for x in range(nk[0]):
            for y in range(nk[1]):
                for z in range(nk[2]):
                    mesh[x % s.nq[0], y % s.nq[1], z % s.nq[2]] += prod[x, y, z]
        sampled = np.fft.ifftn(prod)[::m[0], ::m[1], ::m[2]]
        folded = np.fft.ifftn(mesh) * (np.prod(s.nq) / nkp)
        assert np.max(np.abs(folded - sampled)) < 1e-13 * np.max(np.abs(sampled))


def test_eom_is_a_convolution_over_the_q_mesh():
    p = problem("t3b")
    s = p.spec
    inp = to_inputs(p)
    orc = O.Oracle(inp)
    nd, nk, nkp = s.ndim, s.nk, int(np.prod(s.nk))
    qs = O.generate_q_vol(nk, s.nq) - 1
    rng = np.random.default_rng(5)
    M = rng.standard_normal((len(qs), nd, nd, nd, nd)) + 1j * rng.standard_normal((len(qs), nd, nd, nd, nd))
    G = orc.gk(1).reshape(*nk, nd, nd)                     # G_jk'(k, nu - omega)
    # direct: Sigma_il(k) = sum_q sum_{j,k'} M_q[i, j, l, k'] G_jk'(k - q)
    want = np.zeros((*nk, nd, nd), complex)
    for iq, qk in enumerate(qs):
        shift = kgrid_coords(nk, qk)
        Gs = np.roll(G, shift, axis=(0, 1, 2))             # Gs(k) = G(k - q)
        want += np.einsum("ijlk,xyzjk->xyzil", M[iq], Gs)
    # transform: M^ on the q mesh (q = m a), times G^(p), inverse transform over k
    m = tuple(n // q for n, q in zip(nk, s.nq))
    Mq = np.zeros((*s.nq, nd, nd, nd, nd), complex)
    for iq, qk in enumerate(qs):
        x, y, z = kgrid_coords(nk, qk)
        Mq[x // m[0], y // m[1], z // m[2]] = M[iq]
    Mh = np.fft.fftn(Mq, axes=(0, 1, 2))
    Mh_full = np.tile(Mh, (m[0], m[1], m[2], 1, 1, 1, 1))    # depends on p mod the q mesh
    Gh = np.fft.fftn(G, axes=(0, 1, 2))
    got = np.fft.ifftn(np.einsum("xyzijlk,xyzjk->xyzil", Mh_full, Gh), axes=(0, 1, 2))
    assert np.max(np.abs(got - want)) < 1e-12 * np.max(np.abs(want))


def nopiv_lu32(T):
    A = T.astype(np.complex64).copy()
    for k in range(A.shape[0]):
        A[k + 1:, k] /= A[k, k]
        A[k + 1:, k + 1:] -= np.outer(A[k + 1:, k], A[k, k + 1:])
    return A


def test_bse_matrices_need_no_pivoting_in_the_fp32_factorisation():
    p = problem("t3m")
    s = p.spec
    inp = to_inputs(p)
    orc = O.Oracle(inp)
    out = {k: np.zeros((inp.ndim2, inp.ndim2, 2 * s.iwb + 1), complex)
           for k in ("bubble_loc", "chi_loc_dens", "chi_loc_magn")}
    rng = np.random.default_rng(0)
    for iq, iwb in ((0, 0), (s.nqp - 1, 1)):
        res = orc.point(iq, iwb, orc.local_block(iwb, 1, out))
        for ch in ("A_dens", "A_magn"):
            T = np.asarray(res[ch]).T.copy()               # the factored matrix is the transpose
            LU = nopiv_lu32(T)
            assert np.abs(np.triu(LU)).max() <= 1.5 * np.abs(T).max()       # growth factor
            b = rng.standard_normal((T.shape[0], 9)) + 1j * rng.standard_normal((T.shape[0], 9))
            xt = np.linalg.solve(T, b)

            def solve(r):
                y = sl.solve_triangular(LU, r.astype(np.complex64), lower=True, unit_diagonal=True)
                return sl.solve_triangular(LU, y, lower=False).astype(np.complex128)

            x = solve(b)
            errs = [np.abs(x - xt).max() / np.abs(xt).max()]
            for _ in range(2):                             # FP64 residual, FP32 correction
                x = x + solve(b - T @ x)
                errs.append(np.abs(x - xt).max() / np.abs(xt).max())
            assert errs[0] < 1e-5 and errs[1] < 1e-10 and errs[2] < 1e-13, errs
