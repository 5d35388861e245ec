// chi0 bubble: chi0^q({i,j},{l,k}; nu) = -(beta/nkp) sum_k G_il(k, nu) G_kj(k-q, nu-omega)
// for a batch of q points at one omega -- the k-loop of src/main.F90:646-657
// over accumulate_chi0 (src/one_particle_quant_module.f90:228-290).
//
// One thread block per (nu, point).  Warp w owns the rows i1 = i*nd + j of
// one i (and, for nd > 3, one j); its lanes stride over k, gathering
// G(k, nu) and G(k-q, nu-omega) from the resident G table with 16-byte
// loads, and the partial sums are reduced with warp shuffles.  The kernel
// is bound by the FP64 pipe (81 complex MACs per 288 gathered bytes at
// nd = 3), the table slices it reads stay in L2 across the batch.
#include "ctx.cuh"

template <int ND>
__global__ void __launch_bounds__(32 * ND * (ND <= 3 ? 1 : ND))
k_chi0(DevCtx c, int iwb, const int *__restrict__ qidx, z64 *__restrict__ out, int nnu_all) {
  constexpr int ND2 = ND * ND;
  constexpr int JB = (ND <= 3) ? ND : 1;      // j values per warp
  const int inu = blockIdx.x;                 // 0..nnu_all-1, nu = iwstart + inu
  const int p = blockIdx.y;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int i = warp / (ND / JB);
  const int j0 = (warp % (ND / JB)) * JB;
  const int nu = c.iwstart + inu;
  const int q = qidx[p];
  const z64 *g1t = c.gtab + (size_t)(nu - c.nu_lo) * c.nkp * ND2;
  const z64 *g2t = c.gtab + (size_t)(nu - iwb - c.nu_lo) * c.nkp * ND2;
  const int *kq = c.kq + (size_t)q * c.nkp;

  z64 acc[JB][ND2];
#pragma unroll
  for (int a = 0; a < JB; ++a)
#pragma unroll
    for (int b = 0; b < ND2; ++b) acc[a][b] = make_double2(0.0, 0.0);

  for (int k = lane; k < c.nkp; k += 32) {
    const z64 *g1 = g1t + (size_t)k * ND2;
    const z64 *g2 = g2t + (size_t)__ldg(kq + k) * ND2;
    z64 a1[ND];
#pragma unroll
    for (int l = 0; l < ND; ++l) a1[l] = __ldg(g1 + i + l * ND);      // G_il(k)
    z64 b2[ND][JB];
#pragma unroll
    for (int kk = 0; kk < ND; ++kk)
#pragma unroll
      for (int jj = 0; jj < JB; ++jj) b2[kk][jj] = __ldg(g2 + kk + (j0 + jj) * ND);  // G_kj(k-q)
#pragma unroll
    for (int jj = 0; jj < JB; ++jj)
#pragma unroll
      for (int l = 0; l < ND; ++l)
#pragma unroll
        for (int kk = 0; kk < ND; ++kk) cfma(acc[jj][l * ND + kk], a1[l], b2[kk][jj]);
  }
  // warp reduction
#pragma unroll
  for (int jj = 0; jj < JB; ++jj)
#pragma unroll
    for (int b = 0; b < ND2; ++b) {
      double x = acc[jj][b].x, y = acc[jj][b].y;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        x += __shfl_xor_sync(0xffffffffu, x, o);
        y += __shfl_xor_sync(0xffffffffu, y, o);
      }
      acc[jj][b] = make_double2(x, y);
    }
  // lanes share the stores: output (i1, i2) at i1 + i2*nd2 of block (p, inu)
  z64 *o = out + ((size_t)p * nnu_all + inu) * ND2 * ND2;
  const double f = -c.beta / (double)c.nkp;
#pragma unroll
  for (int jj = 0; jj < JB; ++jj)
#pragma unroll
    for (int b = 0; b < ND2; ++b) {
      if ((jj * ND2 + b) % 32 == lane) {
        int i1 = i * ND + j0 + jj;
        // -beta * sum / nkp; b = l*nd + k is already the column index {l,k}
        o[i1 + b * ND2] = make_double2(acc[jj][b].x * f, acc[jj][b].y * f);
      }
    }
}

cudaError_t launch_chi0(const DevCtx &c, int iwb, const int *qidx, int npts, z64 *chi0_all,
                        int nnu_all, cudaStream_t st) {
  if (npts <= 0) return cudaSuccess;
  dim3 grid(nnu_all, npts);
  switch (c.nd) {
    case 1: k_chi0<1><<<grid, 32, 0, st>>>(c, iwb, qidx, chi0_all, nnu_all); break;
    case 2: k_chi0<2><<<grid, 64, 0, st>>>(c, iwb, qidx, chi0_all, nnu_all); break;
    case 3: k_chi0<3><<<grid, 96, 0, st>>>(c, iwb, qidx, chi0_all, nnu_all); break;
    case 4: k_chi0<4><<<grid, 512, 0, st>>>(c, iwb, qidx, chi0_all, nnu_all); break;
    case 5: k_chi0<5><<<grid, 800, 0, st>>>(c, iwb, qidx, chi0_all, nnu_all); break;
    default: return cudaErrorInvalidValue;
  }
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
