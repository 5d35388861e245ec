// Per-point BSE kernels around the LU:
//   * build  -- A = 1 - blockdiag_nu(chi0^q chi0_loc^-1 - 1) F~ and gamma^q_d
//               (src/main.F90:674-732), written transposed (T = A^T) with the
//               right-hand sides (1 + gamma^w)^T appended as extra columns;
//   * post   -- eta = (1+gamma^w)(A^-1 - 1) from the solve, the chi(q,w)
//               frequency sums of calc_chi_qw (src/main.F90:665-667,766-769;
//               src/susc_module.f90:34-56) and the EOM vertex m_tot
//               (src/eom_module.f90:184-207);
//   * eom    -- Sigma(k, nu) += m_tot G(k-q, nu-w) over a batch of points
//               (src/eom_module.f90:209-230), one owner thread per (k, nu).
#include "ctx.cuh"
#include <algorithm>
#include <type_traits>

// ---------------------------------------------------------------------------
// build: one block per (column tile of A^T rows c, channel, point).
// T(c, r) = delta(c, r) - sum_i3 sw_nu(i1, i3) F~(i3 + nu*nd2, c), r = i1 + nu*nd2
// sw_nu = chi0q(:,:,nu) diag(chi0_loc^-1(nu)) - 1
// ---------------------------------------------------------------------------
template <typename T, int ND2>
__global__ void __launch_bounds__(128)
k_bse_build(DevCtx c, const z64 *__restrict__ chi0q, const z64 *__restrict__ c0inv,
            const z64 *__restrict__ Frow_d, const z64 *__restrict__ Frow_m,
            const z64 *__restrict__ opg_d, const z64 *__restrict__ opg_m, T *Tm, size_t strideM,
            z64 *gammaqd, const int *__restrict__ qidx) {
  __shared__ z64 sw[ND2 * ND2];
  __shared__ z64 sv[ND2 * ND2];   // 2 beta^-2 chi0^q(nu) v(q), density channel with V(q)
  const int N = c.N;
  const int cc = blockIdx.x * blockDim.x + threadIdx.x;
  const int ch = blockIdx.y, p = blockIdx.z;
  const z64 *F = ch == 0 ? Frow_d : Frow_m;
  const z64 *opg = ch == 0 ? opg_d : opg_m;
  T *Tp = Tm + (size_t)(2 * p + ch) * strideM;
  const z64 *c0 = chi0q + (size_t)p * ND2 * ND2 * 2 * c.iwf;
  z64 gq[ND2];
#pragma unroll
  for (int a = 0; a < ND2; ++a) gq[a] = make_double2(0.0, 0.0);
  const bool vterm = c.vq && ch == 0;
  const z64 *vq = vterm ? c.vq + (size_t)qidx[p] * ND2 * ND2 : nullptr;
  z64 og[ND2];                      // (1 + gamma^w_d)(:, cc)
  if (vterm && cc < N)
#pragma unroll
    for (int i3 = 0; i3 < ND2; ++i3) og[i3] = opg_d[i3 + (size_t)cc * ND2];
  for (int dum = 0; dum < 2 * c.iwf; ++dum) {
    __syncthreads();
    for (int e = threadIdx.x; e < ND2 * ND2; e += blockDim.x) {
      int i1 = e % ND2, i3 = e / ND2;
      z64 v = cmul(c0[(size_t)dum * ND2 * ND2 + e], c0inv[dum * ND2 + i3]);
      if (i1 == i3) v.x -= 1.0;
      sw[e] = v;                       // sw(i1, i3) at i1 + i3*nd2
      if (vterm) {                     // src/main.F90:710-719
        z64 t = make_double2(0.0, 0.0);
        for (int m = 0; m < ND2; ++m) cfma(t, c0[(size_t)dum * ND2 * ND2 + i1 + m * ND2], vq[m + i3 * ND2]);
        const double f = 2.0 / (c.beta * c.beta);
        sv[e] = make_double2(f * t.x, f * t.y);
      }
    }
    __syncthreads();
    if (cc < N) {
      z64 f[ND2];
#pragma unroll
      for (int i3 = 0; i3 < ND2; ++i3) f[i3] = F[(size_t)(i3 + dum * ND2) * N + cc];
#pragma unroll
      for (int i1 = 0; i1 < ND2; ++i1) {
        z64 w = make_double2(0.0, 0.0);
#pragma unroll
        for (int i3 = 0; i3 < ND2; ++i3) cfma(w, sw[i1 + i3 * ND2], f[i3]);
        int r = i1 + dum * ND2;
        z64 t = make_double2(-w.x, -w.y);
        if (vterm)
#pragma unroll
          for (int i3 = 0; i3 < ND2; ++i3) cfms(t, sv[i1 + i3 * ND2], og[i3]);
        if (r == cc) t.x += 1.0;
        Tp[cc + (size_t)r * N] = from64<T>(t);
        if (ch == 0) gq[i1] = cadd(gq[i1], w);
      }
    }
  }
  if (cc < N) {
#pragma unroll
    for (int i1 = 0; i1 < ND2; ++i1) Tp[cc + (size_t)(N + i1) * N] = from64<T>(opg[i1 + (size_t)cc * ND2]);
    if (ch == 0 && gammaqd) {
      z64 *g = gammaqd + (size_t)p * ND2 * N;
#pragma unroll
      for (int i1 = 0; i1 < ND2; ++i1) g[i1 + (size_t)cc * ND2] = gq[i1];
    }
  }
}

// Fast build (no V(q) term): one block per (128-column tile, P points) of one
// channel.  A thread owns one column c of T; the F~ rows of each nu block are
// staged into shared memory one nu ahead by cp.async (each thread copies and
// reads only its own column), and sw_nu of the block's points is formed in
// shared memory one nu ahead from chi0^q / chi0_loc^-1 values prefetched into
// registers; one barrier per nu.  F32 selects complex FP32 arithmetic from an
// FP32 copy of F~ -- used for the magnetic channel of the mixed path, whose T
// only feeds the FP32 LU (the FP64 residual of the refinement restores the
// FP64 answer); GQ accumulates gamma^q_d (the density channel, always FP64).
template <int ND2, bool GQ> struct BuildP { static constexpr int P = GQ ? 1 : 2; };

__device__ __forceinline__ void cp_async_bytes(void *smem, const void *gmem, int pred16or8, int nbytes) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  if (pred16or8 == 16)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;" ::"r"(s), "l"(gmem), "r"(nbytes));
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(s), "l"(gmem), "r"(nbytes));
}

template <typename TW, int ND2, bool F32, bool GQ>
__global__ void __launch_bounds__(128)
k_bse_build_fast(DevCtx c, int npts, int ch, const z64 *__restrict__ chi0q, const z64 *__restrict__ c0inv,
                 const void *__restrict__ Fv, const z64 *__restrict__ opg, TW *Tm, size_t strideM, z64 *gammaqd) {
  typedef typename std::conditional<F32, z32, z64>::type A;
  constexpr int P = BuildP<ND2, GQ>::P, ND4 = ND2 * ND2, NE = P * ND4, EPT = (NE + 127) / 128;
  __shared__ __align__(16) A fs[2][ND2][128];
  __shared__ __align__(16) A sws[2][NE];
  const A *F = (const A *)Fv;
  const int N = c.N, nnu = 2 * c.iwf, t = threadIdx.x;
  const int cc = blockIdx.x * 128 + t, p0 = blockIdx.y * P;
  const bool act = cc < N;
  z64 pc[EPT], pinv[EPT];
  auto load_sw = [&](int dum) {
#pragma unroll
    for (int k = 0; k < EPT; ++k) {
      const int e = t + 128 * k;
      if (e < NE) {
        const int pp = e / ND4, el = e % ND4, i3 = el / ND2;
        const int p = p0 + pp;
        pc[k] = p < npts ? chi0q[((size_t)p * nnu + dum) * ND4 + el] : make_double2(0.0, 0.0);
        pinv[k] = c0inv[dum * ND2 + i3];
      }
    }
  };
  auto store_sw = [&](int buf) {
#pragma unroll
    for (int k = 0; k < EPT; ++k) {
      const int e = t + 128 * k;
      if (e < NE) {
        const int el = e % ND4, i1 = el % ND2, i3 = el / ND2;
        z64 v = cmul(pc[k], pinv[k]);
        if (i1 == i3) v.x -= 1.0;
        if constexpr (F32) sws[buf][e] = to32(v);
        else sws[buf][e] = v;
      }
    }
  };
  auto stage_f = [&](int dum, int buf) {
#pragma unroll
    for (int i3 = 0; i3 < ND2; ++i3) {
      const A *g = F + (size_t)(i3 + dum * ND2) * N + (act ? cc : 0);
      cp_async_bytes(&fs[buf][i3][t], g, (int)sizeof(A), act ? (int)sizeof(A) : 0);
    }
    asm volatile("cp.async.commit_group;");
  };
  z64 gq[GQ ? P * ND2 : 1];
  if constexpr (GQ) {
#pragma unroll
    for (int a = 0; a < P * ND2; ++a) gq[a] = make_double2(0.0, 0.0);
  }
  stage_f(0, 0);
  load_sw(0);
  store_sw(0);
  __syncthreads();
  for (int dum = 0; dum < nnu; ++dum) {
    const bool more = dum + 1 < nnu;
    if (more) {
      stage_f(dum + 1, (dum + 1) & 1);
      load_sw(dum + 1);
      asm volatile("cp.async.wait_group 1;" ::: "memory");
    } else {
      asm volatile("cp.async.wait_group 0;" ::: "memory");
    }
    const A *sw = sws[dum & 1];
    A f[ND2];
#pragma unroll
    for (int i3 = 0; i3 < ND2; ++i3) f[i3] = fs[dum & 1][i3][t];
#pragma unroll
    for (int pp = 0; pp < P; ++pp) {
      const int p = p0 + pp;
      if (act && p < npts) {
        TW *Tp = Tm + (size_t)(2 * p + ch) * strideM;
#pragma unroll
        for (int i1 = 0; i1 < ND2; ++i1) {
          A w = cx<A>::make(0, 0);
#pragma unroll
          for (int i3 = 0; i3 < ND2; ++i3) cfma(w, sw[pp * ND4 + i1 + i3 * ND2], f[i3]);
          const int r = i1 + dum * ND2;
          A tv = cx<A>::make(-w.x, -w.y);
          if (r == cc) tv.x += 1;
          if constexpr (F32) Tp[cc + (size_t)r * N] = tv;
          else Tp[cc + (size_t)r * N] = from64<TW>(tv);
          if constexpr (GQ) gq[pp * ND2 + i1] = cadd(gq[pp * ND2 + i1], w);
        }
      }
    }
    if (more) store_sw((dum + 1) & 1);
    __syncthreads();
  }
  if (!act) return;
#pragma unroll
  for (int pp = 0; pp < P; ++pp) {
    const int p = p0 + pp;
    if (p >= npts) continue;
    TW *Tp = Tm + (size_t)(2 * p + ch) * strideM;
#pragma unroll
    for (int i1 = 0; i1 < ND2; ++i1) Tp[cc + (size_t)(N + i1) * N] = from64<TW>(opg[i1 + (size_t)cc * ND2]);
    if constexpr (GQ) {
      if (gammaqd) {
        z64 *g = gammaqd + (size_t)p * ND2 * N;
#pragma unroll
        for (int i1 = 0; i1 < ND2; ++i1) g[i1 + (size_t)cc * ND2] = gq[pp * ND2 + i1];
      }
    }
  }
}

__global__ void k_to32(size_t n, const z64 *__restrict__ x, z32 *__restrict__ y) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    y[i] = to32(x[i]);
}

cudaError_t launch_to32(size_t n, const z64 *x, z32 *y, cudaStream_t st) {
  if (!n) return cudaSuccess;
  k_to32<<<(unsigned)std::min<size_t>(cdiv_u(n, 256), 4096), 256, 0, st>>>(n, x, y);
  return ADGA_LAUNCH_CHECK();
}

template <typename T>
cudaError_t launch_bse_build(const DevCtx &c, int npts, const z64 *chi0q, const z64 *c0inv,
                             const z64 *Frow_d, const z64 *Frow_m, const z64 *opg_d,
                             const z64 *opg_m, T *Tmat, size_t strideM, z64 *gammaqd,
                             const int *qidx, cudaStream_t st, const z32 *F32_m) {
  if (npts <= 0) return cudaSuccess;
  if (!c.vq && c.nd2 <= 9) {
    cudaError_t e = cudaSuccess;
#define FAST(NDD)                                                                                          \
  {                                                                                                        \
    dim3 g(cdiv_u(c.N, 128), cdiv_u(npts, BuildP<NDD, true>::P));                                         \
    k_bse_build_fast<T, NDD, false, true><<<g, 128, 0, st>>>(c, npts, 0, chi0q, c0inv, Frow_d, opg_d,      \
                                                             Tmat, strideM, gammaqd);                      \
    if ((e = ADGA_LAUNCH_CHECK()) != cudaSuccess) return e;                                                \
    g.y = cdiv_u(npts, BuildP<NDD, false>::P);                                                             \
    bool done = false;                                                                                     \
    if constexpr (std::is_same<T, z32>::value) {                                                           \
      if (F32_m) {                                                                                         \
        k_bse_build_fast<T, NDD, true, false><<<g, 128, 0, st>>>(c, npts, 1, chi0q, c0inv, F32_m, opg_m,   \
                                                                 Tmat, strideM, nullptr);                  \
        done = true;                                                                                       \
      }                                                                                                    \
    }                                                                                                      \
    if (!done)                                                                                             \
      k_bse_build_fast<T, NDD, false, false><<<g, 128, 0, st>>>(c, npts, 1, chi0q, c0inv, Frow_m, opg_m,   \
                                                                Tmat, strideM, nullptr);                   \
  }
    switch (c.nd2) {      // nd <= 3; larger orbital counts take the general kernel below
      case 1: FAST(1); break;
      case 4: FAST(4); break;
      case 9: FAST(9); break;
    }
#undef FAST
    if (c.nd2 <= 9) return ADGA_LAUNCH_CHECK();
  }
  dim3 grid(cdiv_u(c.N, 128), 2, npts);
#define BUILD(NDD)                                                                            \
  k_bse_build<T, NDD><<<grid, 128, 0, st>>>(c, chi0q, c0inv, Frow_d, Frow_m, opg_d, opg_m,     \
                                            Tmat, strideM, gammaqd, qidx)
  switch (c.nd2) {
    case 1: BUILD(1); break;
    case 4: BUILD(4); break;
    case 9: BUILD(9); break;
    case 16: BUILD(16); break;
    case 25: BUILD(25); break;
    default: return cudaErrorInvalidValue;
  }
#undef BUILD
  return ADGA_LAUNCH_CHECK();
}
template cudaError_t launch_bse_build<z64>(const DevCtx &, int, const z64 *, const z64 *,
                                           const z64 *, const z64 *, const z64 *, const z64 *,
                                           z64 *, size_t, z64 *, const int *, cudaStream_t, const z32 *);
template cudaError_t launch_bse_build<z32>(const DevCtx &, int, const z64 *, const z64 *,
                                           const z64 *, const z64 *, const z64 *, const z64 *,
                                           z32 *, size_t, z64 *, const int *, cudaStream_t, const z32 *);

// ---------------------------------------------------------------------------
// post: one block per point.
//   X_ch(c, i1) (column-major, ld ldX) = ((1+gamma^w) A^-1)^T  -> eta = X^T - (1+gamma^w)
//   chi_ch = beta^-2 sum gamma (chi0q - chi0w) + beta^-2 sum eta chi0q
//   m_tot(:, nu >= 0 half) = -(u - u~/2) eta_d/(beta nqp) + 1.5 u~ eta_m/(beta nqp)
//                            + u gamma^q_d/(beta nqp)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
k_post(DevCtx c, const z64 *__restrict__ X, size_t sp, size_t sc, int ldX, const z64 *__restrict__ opg_d,
       const z64 *__restrict__ opg_m, const z64 *__restrict__ gam_d, const z64 *__restrict__ gam_m,
       const z64 *__restrict__ gammaqd, const z64 *__restrict__ chi0q, const z64 *__restrict__ c0w,
       z64 *chi_qw_d, z64 *chi_qw_m, z64 *mtot, z64 *etad, z64 *etam, const int *__restrict__ qidx) {
  const int p = blockIdx.x;
  const int N = c.N, nd2 = c.nd2, iwf = c.iwf;
  const size_t nd2N = (size_t)nd2 * N;
  z64 *ed = etad + p * nd2N, *em = etam + p * nd2N;
  const z64 *Xd = X + (size_t)p * sp, *Xm = Xd + sc;
  // 1. eta
  for (size_t e = threadIdx.x; e < nd2N; e += blockDim.x) {
    int i1 = (int)(e % nd2), cc = (int)(e / nd2);
    ed[e] = csub(Xd[cc + (size_t)i1 * ldX], opg_d[e]);
    em[e] = csub(Xm[cc + (size_t)i1 * ldX], opg_m[e]);
  }
  __syncthreads();
  const z64 *c0 = chi0q + (size_t)p * nd2 * nd2 * 2 * iwf;
  const double b2 = c.beta * c.beta;
  // 2. chi sums: eight lanes per (i1, i2, channel), lane l of the group summing the
  //    frequencies dum = l mod 8, then a shuffle reduction (every lane of a warp
  //    runs the same rounds)
  {
    const int l8 = threadIdx.x & 7, grp = threadIdx.x >> 3, ngrp = blockDim.x >> 3;
    const int total = 2 * nd2 * nd2;
    for (int base = 0; base < total; base += ngrp) {
      const int t = base + grp;
      z64 s1 = make_double2(0.0, 0.0), s2 = make_double2(0.0, 0.0);
      int ch = 0, e = 0;
      if (t < total) {
        ch = t / (nd2 * nd2);
        e = t % (nd2 * nd2);
        const int i1 = e % nd2, i2 = e / nd2;
        const z64 *g = ch ? gam_m : gam_d;
        const z64 *et = ch ? em : ed;
        for (int dum = l8; dum < 2 * iwf; dum += 8) {
          const z64 *cq = c0 + (size_t)dum * nd2 * nd2 + (size_t)i2 * nd2;
          for (int i3 = 0; i3 < nd2; ++i3) {
            const size_t col = (size_t)(i3 + dum * nd2) * nd2;
            const z64 q = cq[i3];
            z64 nl = q;
            if (i3 == i2) nl = csub(q, c0w[dum * nd2 + i2]);
            cfma(s1, g[i1 + col], nl);
            cfma(s2, et[i1 + col], q);
          }
        }
      }
#pragma unroll
      for (int o = 4; o > 0; o >>= 1) {
        s1.x += __shfl_xor_sync(0xffffffffu, s1.x, o);
        s1.y += __shfl_xor_sync(0xffffffffu, s1.y, o);
        s2.x += __shfl_xor_sync(0xffffffffu, s2.x, o);
        s2.y += __shfl_xor_sync(0xffffffffu, s2.y, o);
      }
      if (t < total && l8 == 0) {
        z64 *out = (ch ? chi_qw_m : chi_qw_d) + (size_t)p * nd2 * nd2 + e;
        z64 v = make_double2(s1.x / b2, s1.y / b2);
        *out = cadd(v, make_double2(s2.x / b2, s2.y / b2));
      }
    }
  }
  // 3. m_tot for the nu >= 0 half of the columns
  if (mtot) {
    const double inv = 1.0 / c.beta / (double)c.nqp;
    // V(q) terms of m_tot (src/eom_module.f90:187-205)
    const z64 *vq = (c.vq && qidx) ? c.vq + (size_t)qidx[p] * nd2 * nd2 : nullptr;
    const z64 *gq = gammaqd + (size_t)p * nd2N;
    z64 *m = mtot + (size_t)p * nd2 * iwf * nd2;
    for (int t = threadIdx.x; t < nd2 * iwf * nd2; t += blockDim.x) {
      int i1 = t % nd2, cl = t / nd2;          // local column
      size_t col = (size_t)(cl + iwf * nd2) * nd2;
      z64 a1 = make_double2(0.0, 0.0), a2 = a1, a3 = a1, a4 = a1;
      for (int i3 = 0; i3 < nd2; ++i3) {
        z64 uu = c.u[i1 + i3 * nd2], tt = c.ut[i1 + i3 * nd2];
        z64 uw = make_double2(uu.x - 0.5 * tt.x, uu.y - 0.5 * tt.y);
        if (vq) uw = cadd(vq[i1 + i3 * nd2], uw);       // u_work = v + u - u~/2
        cfma(a1, uw, ed[i3 + col]);
        cfma(a2, tt, em[i3 + col]);
        cfma(a3, uu, gq[i3 + col]);
        if (vq) cfma(a4, vq[i1 + i3 * nd2], gam_d[i3 + col]);   // v gamma^w_d
      }
      z64 v = cscale(a1, -inv);
      v = cadd(cscale(a2, 1.5 * inv), v);
      v = cadd(cscale(a3, inv), v);
      if (vq) v = cadd(cscale(a4, -inv), v);
      m[t] = v;
    }
  }
}

cudaError_t launch_post(const DevCtx &c, int npts, const z64 *X, size_t sp, size_t sc, int ldX,
                        const z64 *opg_d, const z64 *opg_m, const z64 *gam_d, const z64 *gam_m,
                        const z64 *gammaqd, const z64 *chi0q, const z64 *c0w, z64 *chi_qw_d,
                        z64 *chi_qw_m, z64 *mtot, z64 *etad, z64 *etam, const int *qidx, cudaStream_t st) {
  if (npts <= 0) return cudaSuccess;
  k_post<<<npts, 256, 0, st>>>(c, X, sp, sc, ldX, opg_d, opg_m, gam_d, gam_m, gammaqd, chi0q, c0w,
                               chi_qw_d, chi_qw_m, mtot, etad, etam, qidx);
  return ADGA_LAUNCH_CHECK();
}

// ---------------------------------------------------------------------------
// eom: Sigma(i,l,nu,k) += sum_p sum_{k',j} m_tot_p({j,i},{k',l,nu}) G_jk'(k - q_p, nu - w)
// One block per (k tile, nu >= 0); the m_tot slice of each point is staged in
// shared memory, G is gathered from the resident table.  Summation order per
// element follows the reference: points in order, k' outer, j inner.
// ---------------------------------------------------------------------------
template <int ND>
__global__ void __launch_bounds__(128)
k_eom_dyn(DevCtx c, int iwb, const int *__restrict__ qidx, int npts, const z64 *__restrict__ mtot,
          z64 *sigma) {
  constexpr int ND2 = ND * ND;
  __shared__ z64 M[ND2 * ND2];
  const int nu = blockIdx.y;                  // 0..iwf-1
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int iwf = c.iwf;
  const bool act = k < c.nkp_eom;
  z64 acc[ND2];
  z64 *so = sigma + ((size_t)k * 2 * iwf + nu + iwf) * ND2;
#pragma unroll
  for (int a = 0; a < ND2; ++a) acc[a] = act ? so[a] : make_double2(0.0, 0.0);
  const z64 *gt = c.gtab + (size_t)(nu - iwb - c.nu_lo) * c.nkp * ND2;
  for (int p = 0; p < npts; ++p) {
    __syncthreads();
    const z64 *mp = mtot + (size_t)p * ND2 * iwf * ND2 + (size_t)nu * ND2 * ND2;
    for (int e = threadIdx.x; e < ND2 * ND2; e += blockDim.x) M[e] = mp[e];
    __syncthreads();
    if (act) {
      int kk = c.kqe[k + (size_t)qidx[p] * c.nkp_eom];
      const z64 *g = gt + (size_t)kk * ND2;
      z64 G[ND2];
#pragma unroll
      for (int a = 0; a < ND2; ++a) G[a] = __ldg(g + a);
#pragma unroll
      for (int l = 0; l < ND; ++l)
#pragma unroll
        for (int k2 = 0; k2 < ND; ++k2)
#pragma unroll
          for (int i = 0; i < ND; ++i)
#pragma unroll
            for (int j = 0; j < ND; ++j)
              cfma(acc[i + l * ND], M[(i * ND + j) + (l * ND + k2) * ND2], G[j + k2 * ND]);
    }
  }
  if (act) {
#pragma unroll
    for (int a = 0; a < ND2; ++a) so[a] = acc[a];
  }
}

cudaError_t launch_eom_dynamic(const DevCtx &c, int iwb, const int *qidx, int npts,
                               const z64 *mtot, z64 *sigma_nl, cudaStream_t st) {
  if (npts <= 0) return cudaSuccess;
  if (c.dft.ghat && npts >= c.dft.min_points)
    return launch_eom_dft(c, iwb, qidx, npts, mtot, c.dft.ghat, sigma_nl, st);
  dim3 grid(cdiv_u(c.nkp_eom, 128), c.iwf);
  switch (c.nd) {
    case 1: k_eom_dyn<1><<<grid, 128, 0, st>>>(c, iwb, qidx, npts, mtot, sigma_nl); break;
    case 2: k_eom_dyn<2><<<grid, 128, 0, st>>>(c, iwb, qidx, npts, mtot, sigma_nl); break;
    case 3: k_eom_dyn<3><<<grid, 128, 0, st>>>(c, iwb, qidx, npts, mtot, sigma_nl); break;
    case 4: k_eom_dyn<4><<<grid, 128, 0, st>>>(c, iwb, qidx, npts, mtot, sigma_nl); break;
    case 5: k_eom_dyn<5><<<grid, 128, 0, st>>>(c, iwb, qidx, npts, mtot, sigma_nl); break;
    default: return cudaErrorInvalidValue;
  }
  return ADGA_LAUNCH_CHECK();
}
