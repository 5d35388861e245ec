// chi0 bubble: chi0^q({i,j},{l,k}; nu) = -(beta/nkp) sum_k G_il(k, nu) G_kj(k-q, nu-omega)
// for a batch of q points at one omega -- the k-loop of src/main.F90:646-657
// over accumulate_chi0 (src/one_particle_quant_module.f90:228-290).
//
// The kernel is bound by the FP64 pipe (nd2 complex MACs per gathered
// 16-byte G(k-q) value); the G-table slices it reads stay in L2 across the
// batch.
#include "ctx.cuh"

// Thread (q, b) of a CTA owns one column b = (k', j) of G(k-q, nu-omega) and
// one point q, and accumulates the nd2 products with every entry a = (i, l)
// of G(k, nu) over k.  G(k, nu) is staged in shared memory in chunks of KC
// k-points and read as broadcasts; the k-q indices of the CTA's points are
// staged beside it.  Each gathered G(k-q) value feeds nd2 complex FMAs.
template <int ND, int QG>
__global__ void __launch_bounds__(QG * ND * ND)
k_chi0(DevCtx c, int iwb, const int *__restrict__ qidx, int npts, z64 *__restrict__ out, int nnu_all,
       const z64 *__restrict__ g2tab) {
  constexpr int ND2 = ND * ND, KC = 64, NTH = QG * ND2;
  __shared__ z64 g1s[KC][ND2];
  __shared__ int kqs[KC][QG];
  const int inu = blockIdx.x, p0 = blockIdx.y * QG;
  const int t = threadIdx.x, ql = t / ND2, bcol = t % ND2;
  const int p = p0 + ql;
  const bool act = p < npts;
  const int nu = c.iwstart + inu;
  const z64 *g1t = c.gtab + (size_t)(nu - c.nu_lo) * c.nkp * ND2;
  const z64 *g2t = (g2tab ? g2tab : c.gtab) + (size_t)(nu - iwb - c.nu_lo) * c.nkp * ND2;
  z64 acc[ND2];
#pragma unroll
  for (int a = 0; a < ND2; ++a) acc[a] = make_double2(0.0, 0.0);
  for (int k0 = 0; k0 < c.nkp; k0 += KC) {
    const int kc = min(KC, c.nkp - k0);
    __syncthreads();
    for (int e = t; e < kc * ND2; e += NTH) g1s[e / ND2][e % ND2] = __ldg(g1t + (size_t)k0 * ND2 + e);
    for (int e = t; e < kc * QG; e += NTH) {
      const int q_l = e / kc, kk = e % kc, pp = p0 + q_l;
      kqs[kk][q_l] = pp < npts ? __ldg(c.kq + (k0 + kk) + (size_t)qidx[pp] * c.nkp) : 0;
    }
    __syncthreads();
    if (act) {
#pragma unroll 4
      for (int kk = 0; kk < kc; ++kk) {
        const z64 g2 = __ldg(g2t + (size_t)kqs[kk][ql] * ND2 + bcol);
#pragma unroll
        for (int a = 0; a < ND2; ++a) cfma(acc[a], g1s[kk][a], g2);
      }
    }
  }
  if (!act) return;
  // a = i + l*nd (G_il(k)), bcol = k' + j*nd (G_k'j(k-q)): chi0({i,j},{l,k'})
  z64 *o = out + ((size_t)p * nnu_all + inu) * ND2 * ND2;
  const double f = -c.beta / (double)c.nkp;
  const int kp = bcol % ND, j = bcol / ND;
#pragma unroll
  for (int a = 0; a < ND2; ++a) {
    const int i = a % ND, l = a / ND;
    o[(i * ND + j) + (l * ND + kp) * ND2] = make_double2(acc[a].x * f, acc[a].y * f);
  }
}

cudaError_t launch_chi0(const DevCtx &c, int iwb, const int *qidx, int npts, z64 *chi0_all,
                        int nnu_all, cudaStream_t st, const z64 *g2tab, const z64 *g2hat) {
  if (npts <= 0) return cudaSuccess;
  if (c.dft.ghat && npts >= c.dft.min_points && (!g2tab || g2hat))
    return launch_chi0_dft(c, iwb, qidx, npts, chi0_all, nnu_all, c.dft.ghat, g2tab ? g2hat : c.dft.ghat, st);
#define CHI0(NDD, QGG)                                                                      \
  k_chi0<NDD, QGG><<<dim3(nnu_all, cdiv_u(npts, QGG)), QGG * NDD * NDD, 0, st>>>(c, iwb, qidx, \
                                                                                npts, chi0_all, nnu_all, g2tab)
  switch (c.nd) {
    case 1: CHI0(1, 128); break;
    case 2: CHI0(2, 32); break;
    case 3: CHI0(3, 16); break;
    case 4: CHI0(4, 8); break;
    case 5: CHI0(5, 8); break;
    default: return cudaErrorInvalidValue;
  }
#undef CHI0
  return ADGA_LAUNCH_CHECK();
}

// chi0q (small box) and bubble_nl = sum_{iwstart..iwstop} chi0 / beta^2 -
// bubble_loc_tmp (src/main.F90:655-663).  One thread per (i1,i2,point).
__global__ void k_chi0_finish(DevCtx c, const z64 *all, int nnu_all, int npts, const z64 *bub_tmp,
                              z64 *chi0q, z64 *bub_nl) {
  size_t nd4 = (size_t)c.nd2 * c.nd2;
  size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (idx >= nd4 * npts) return;
  size_t e = idx % nd4, p = idx / nd4;
  const z64 *a = all + p * nnu_all * nd4 + e;
  z64 s = make_double2(0.0, 0.0);
  int off = -c.iwf - c.iwstart;   // index of nu = -iwf in the full list
  for (int inu = 0; inu < nnu_all; ++inu) {
    z64 v = a[(size_t)inu * nd4];
    s = cadd(s, v);
    int ism = inu - off;
    if (chi0q && ism >= 0 && ism < 2 * c.iwf) chi0q[(p * 2 * c.iwf + ism) * nd4 + e] = v;
  }
  if (bub_nl) {
    double b2 = c.beta * c.beta;
    z64 t = bub_tmp[e];
    bub_nl[p * nd4 + e] = make_double2(s.x / b2 - t.x, s.y / b2 - t.y);
  }
}

cudaError_t launch_chi0_finish(const DevCtx &c, const z64 *chi0_all, int nnu_all, int npts,
                               const z64 *bubloc_tmp, z64 *chi0q, z64 *bubble_nl, cudaStream_t st) {
  size_t total = (size_t)c.nd2 * c.nd2 * npts;
  if (!total) return cudaSuccess;
  k_chi0_finish<<<cdiv_u(total, 256), 256, 0, st>>>(c, chi0_all, nnu_all, npts, bubloc_tmp,
                                                    chi0q, bubble_nl);
  return ADGA_LAUNCH_CHECK();
}
