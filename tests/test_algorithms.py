"""CPU checks of algorithmic choices of the GPU path (numpy restatements, no
GPU), the first two against the oracle's own data:

* the bubble and the EOM are cyclic correlations / convolutions over the k
  mesh, so they equal DFT products, and sampling the inverse transform on the
  q sub-mesh equals folding the products onto it (the transform path of
  k_dft.cu);
* the transposed BSE matrices 1 - D F~ factor without row interchanges with
  growth factor ~1, and that unpivoted FP32 LU contracts FP64 iterative
  refinement as fast as a pivoted one (the mixed path's factorisation);
* the trailing update's six bf16 segment products, in the tensor-core
  kernel's order and slot layout, form the 3-term complex product and free
  their operand slots in fill order;
* the diagonal-block kernel's recursive doubling gives both triangular
  inverses.
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


def _bf16(x):
    """float32 -> the nearest bfloat16 (ties to even), returned as float32."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32)
    u = (u + (0x7FFF + ((u >> 16) & 1))) & np.uint32(0xFFFF0000)
    return u.view(np.float32)


def test_trailing_update_segment_products_form_the_complex_product():
    """The tensor-core trailing update (k_tc.cu, k_tc_persist) stages per step
    A = [Lr_hi, Li_hi, Lr_lo, Li_lo] (rows of L21) and B = [Ur_hi, -Ui_hi, Ur_lo,
    -Ui_lo] (columns of U12), loads them as slot pairs [B2 B3] [A0 A1] [B0 B1]
    [A2 A3] and runs six products in the order j = 2, 3, 0, 1, 4, 5: A segment a
    times B segment b into the real part and B segment b ^ 1 (negated for even b)
    into the imaginary part.  Together they are the 3-term bf16 split of
    L U, (hi, hi) + (hi, lo) + (lo, hi), and every slot is released after its
    last product in the order the slots were filled."""
    rng = np.random.default_rng(3)
    m, k, n = 24, 64, 20
    L = (rng.standard_normal((m, k)) + 1j * rng.standard_normal((m, k))).astype(np.complex64)
    U = (rng.standard_normal((k, n)) + 1j * rng.standard_normal((k, n))).astype(np.complex64)
    split = lambda x: (_bf16(x), _bf16(x - _bf16(x)))
    (lrh, lrl), (lih, lil) = split(L.real), split(L.imag)
    (urh, url), (uih, uil) = split(U.real), split(U.imag)
    A = [lrh, lih, lrl, lil]                              # m x k each
    B = [urh.T, -uih.T, url.T, -uil.T]                    # n x k each (K-major rows)
    # kernel order: (j, A segment, B segment of the real part); imaginary part from b ^ 1
    seg_a = {0: 0, 1: 1, 2: 0, 3: 1, 4: 2, 5: 3}
    seg_b = {0: 0, 1: 1, 2: 2, 3: 3, 4: 0, 5: 1}
    re = np.zeros((m, n))
    im = np.zeros((m, n))
    for j in (2, 3, 0, 1, 4, 5):
        a, b = seg_a[j], seg_b[j]
        sign = -1.0 if b % 2 == 0 else 1.0
        re += A[a].astype(np.float64) @ B[b].T.astype(np.float64)
        im += sign * (A[a].astype(np.float64) @ B[b ^ 1].T.astype(np.float64))
    want = L.astype(np.complex128) @ U.astype(np.complex128)
    scale = np.abs(L).astype(np.float64) @ np.abs(U).astype(np.float64)
    assert np.max(np.abs(re + 1j * im - want) / scale) < 2.0 ** -15
    # slots: fill order 0..3 holds [B2 B3], [A0 A1], [B0 B1], [A2 A3]; a slot is released
    # after the last product that reads it
    slot_of = {("B", 2): 0, ("B", 3): 0, ("A", 0): 1, ("A", 1): 1, ("B", 0): 2, ("B", 1): 2,
               ("A", 2): 3, ("A", 3): 3}
    last = {}
    for step, j in enumerate((2, 3, 0, 1, 4, 5)):
        a, b = seg_a[j], seg_b[j]
        for key in (("A", a), ("B", b), ("B", b ^ 1)):
            last[slot_of[key]] = step
    releases = sorted(last, key=lambda s: (last[s], s))
    assert releases == [0, 1, 2, 3]


def test_triangular_inverses_by_recursive_doubling():
    """The diagonal-block kernel (k_lu.cu, k_diag_inv) inverts the unit lower and
    the upper factor of the 64 x 64 block from their 16 x 16 diagonal blocks by
    two doubling levels, X10 = -X11 (L10 X00) for L and Y01 = -Y00 (U01 Y11) for
    U, 16 -> 32 -> 64."""
    rng = np.random.default_rng(5)
    n = 64
    A = np.eye(n) + 0.1 * (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))
    D = A.copy()                                           # unpivoted LU, as the kernel factors
    for j in range(n):
        D[j + 1:, j] /= D[j, j]
        D[j + 1:, j + 1:] -= np.outer(D[j + 1:, j], D[j, j + 1:])
    Lf, Uf = np.tril(D, -1) + np.eye(n), np.triu(D)
    assert np.allclose(Lf @ Uf, A)
    X = np.zeros((n, n), complex)                          # L^-1 and U^-1 built blockwise
    Y = np.zeros((n, n), complex)
    for o in range(0, n, 16):
        X[o:o + 16, o:o + 16] = np.linalg.inv(Lf[o:o + 16, o:o + 16])
        Y[o:o + 16, o:o + 16] = np.linalg.inv(Uf[o:o + 16, o:o + 16])
    for h in (16, 32):
        for o in range(0, n, 2 * h):
            lo, hi = slice(o, o + h), slice(o + h, o + 2 * h)
            X[hi, lo] = -X[hi, hi] @ (Lf[hi, lo] @ X[lo, lo])
            Y[lo, hi] = -Y[lo, lo] @ (Uf[lo, hi] @ Y[hi, hi])
    assert np.max(np.abs(X - np.linalg.inv(Lf))) < 1e-12
    assert np.max(np.abs(Y - np.linalg.inv(Uf))) < 1e-12
