// Post-loop assembly of the DGA self-energy (src/main.F90:869-890):
//   add_siw_dmft     Sigma(i,i,nu,k) += siw(nu,i)            (src/eom_module.f90:237-251)
//   get_sigma_g_loc  sigma_loc(nu) = <Sigma(nu,k)>_k and
//                    gloc(nu) = <(i nu + mu - H(k) - dc - Sigma(nu,k))^-1>_k with the
//                    DGA Sigma inside the vertex box and the DMFT siw outside,
//                    gloc(-nu-1) = gloc(nu)^dagger   (src/one_particle_quant_module.f90:129-187)
//   get_ndga         n(k) = 2/beta sum_{nu>=0} Re G(k,nu) + 1/2 on the diagonal and its
//                    k average (src/one_particle_quant_module.f90:344-394, get_gkiw_dga :106-126)
// Reductions over k and nu run in a fixed order (per-thread partial sums, then
// a fixed tree), so results do not depend on scheduling.
#include "ctx.cuh"
#include <algorithm>
#include "ginv.cuh"

#define PL_MAXND GINV_MAXND

// G(k, nu) with the self-energy sig (nd x nd, column-major), or diag(siw(nu)) when sig is null
__device__ __forceinline__ void pl_gk(const DevCtx &c, int kfull, int nu, const z64 *sig, z64 *a) {
  const int nd = c.nd;
  const z64 *h = c.hk + (size_t)kfull * c.nd2;
  for (int e = 0; e < nd * nd; ++e) a[e] = cneg(h[e]);
  if (sig)
    for (int e = 0; e < nd * nd; ++e) a[e] = csub(a[e], sig[e]);
  const double w = c.iw[nu + c.iwmax];
  for (int i = 0; i < nd; ++i) {
    z64 d = make_double2(c.mu, w);
    d = csub(d, h[i + i * nd]);
    d = csub(d, c.dc[2 * i]);
    d = csub(d, sig ? sig[i + i * nd] : c.siw[(nu + c.iwmax) + i * 2 * c.iwmax]);
    a[i + i * nd] = d;
  }
  ginv_small(nd, a);
}

__global__ void k_add_siw(DevCtx c, z64 *sig, int nk) {
  const size_t n = (size_t)c.nd * 2 * c.iwf * nk;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(idx % c.nd);
    const size_t rest = idx / c.nd;
    const int nu = (int)(rest % (2 * c.iwf)) - c.iwf;
    const size_t k = rest / (2 * c.iwf);
    z64 &s = sig[(size_t)(i + i * c.nd) + c.nd2 * ((size_t)(nu + c.iwf) + 2 * (size_t)c.iwf * k)];
    s = cadd(s, c.siw[(nu + c.iwmax) + i * 2 * c.iwmax]);
  }
}

// block-wide sum of v over the 256 threads (fixed order), result valid in thread 0
__device__ __forceinline__ z64 pl_block_sum(z64 v, z64 *red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    v.x += __shfl_down_sync(0xffffffffu, v.x, o);
    v.y += __shfl_down_sync(0xffffffffu, v.y, o);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  z64 s = make_double2(0.0, 0.0);
  if (threadIdx.x == 0)
    for (int w = 0; w < 8; ++w) s = cadd(s, red[w]);
  return s;
}

// sigma_loc(i,j,nu) = 1/nkp sum_k Sigma(i,j,nu,k): one block per (element, nu)
__global__ void __launch_bounds__(256) k_sigma_loc(DevCtx c, const z64 *sig, z64 *sig_loc) {
  __shared__ z64 red[8];
  const int e = blockIdx.x % c.nd2, inu = blockIdx.x / c.nd2;
  z64 acc = make_double2(0.0, 0.0);
  for (int k = threadIdx.x; k < c.nkp; k += 256)
    acc = cadd(acc, sig[(size_t)e + c.nd2 * ((size_t)inu + 2 * (size_t)c.iwf * k)]);
  const z64 s = pl_block_sum(acc, red);
  if (threadIdx.x == 0) sig_loc[e + c.nd2 * inu] = make_double2(s.x / c.nkp, s.y / c.nkp);
}

// gloc(nu, i, j) for nu = 0..iwmax-1 (one block per nu), mirrored to -nu-1
__global__ void __launch_bounds__(256) k_gloc(DevCtx c, const z64 *sig, z64 *gloc) {
  __shared__ z64 red[8];
  const int nu = blockIdx.x, nd = c.nd, nd2 = c.nd2;
  z64 acc[PL_MAXND * PL_MAXND];
  for (int e = 0; e < nd2; ++e) acc[e] = make_double2(0.0, 0.0);
  for (int k = threadIdx.x; k < c.nkp; k += 256) {
    z64 a[PL_MAXND * PL_MAXND];
    const z64 *s = nu < c.iwf ? sig + (size_t)nd2 * ((size_t)(nu + c.iwf) + 2 * (size_t)c.iwf * k) : nullptr;
    pl_gk(c, k, nu, s, a);
    for (int e = 0; e < nd2; ++e) acc[e] = cadd(acc[e], a[e]);
  }
  const size_t n2w = 2 * (size_t)c.iwmax;
  for (int e = 0; e < nd2; ++e) {
    const z64 v = pl_block_sum(acc[e], red);
    if (threadIdx.x == 0) {
      const int i = e % nd, j = e / nd;
      const z64 g = make_double2(v.x / c.nkp, v.y / c.nkp);
      gloc[(size_t)(nu + c.iwmax) + n2w * (i + (size_t)nd * j)] = g;
      // G(-nu-1) = G(nu)^dagger: element (j, i) of the mirror is conj(G(i, j))
      gloc[(size_t)(-nu - 1 + c.iwmax) + n2w * (j + (size_t)nd * i)] = make_double2(g.x, -g.y);
    }
  }
}

// occupation n(ik, i, j) = 2/beta sum_{nu>=0} Re G(k, nu) + 1/2 delta_ij over nk k-points
// (Fortran order, complex with zero imaginary part): n_dga_k with the DGA Sigma inside
// the box (get_ndga), or n_fock with the DMFT siw everywhere when sig is null (get_nfock,
// src/one_particle_quant_module.f90:316-342)
__global__ void __launch_bounds__(128) k_occ(DevCtx c, int nkk, const int *keom, const z64 *sig, z64 *nk) {
  const int ik = blockIdx.x * blockDim.x + threadIdx.x;
  if (ik >= nkk) return;
  const int nd = c.nd, nd2 = c.nd2;
  const int kfull = keom ? keom[ik] - 1 : ik;
  double acc[PL_MAXND * PL_MAXND];
  for (int e = 0; e < nd2; ++e) acc[e] = 0.0;
  for (int nu = 0; nu < c.iwmax; ++nu) {
    z64 a[PL_MAXND * PL_MAXND];
    const z64 *s = (sig && nu < c.iwf) ? sig + (size_t)nd2 * ((size_t)(nu + c.iwf) + 2 * (size_t)c.iwf * ik) : nullptr;
    pl_gk(c, kfull, nu, s, a);
    for (int e = 0; e < nd2; ++e) acc[e] += a[e].x;
  }
  for (int e = 0; e < nd2; ++e) {
    const int i = e % nd, j = e / nd;
    double v = 2.0 * acc[e] / c.beta;
    if (i == j) v += 0.5;
    nk[(size_t)ik + (size_t)nkk * e] = make_double2(v, 0.0);
  }
}

// n_dga(i) = 1/nkp_eom sum_k n_dga_k(k, i, i): one block per orbital
__global__ void __launch_bounds__(256) k_ndga(DevCtx c, const z64 *nk, z64 *n) {
  __shared__ z64 red[8];
  const int i = blockIdx.x;
  z64 acc = make_double2(0.0, 0.0);
  for (int k = threadIdx.x; k < c.nkp_eom; k += 256)
    acc = cadd(acc, nk[(size_t)k + (size_t)c.nkp_eom * (i + (size_t)c.nd * i)]);
  const z64 s = pl_block_sum(acc, red);
  if (threadIdx.x == 0) n[i] = make_double2(s.x / c.nkp_eom, s.y / c.nkp_eom);
}

cudaError_t launch_post_loop(const DevCtx &c, const int *keom, z64 *sig, z64 *sig_loc, z64 *gloc,
                             z64 *n_dga_k, z64 *n_dga, cudaStream_t st) {
  if (c.nd > PL_MAXND) return cudaErrorInvalidValue;
  const size_t n = (size_t)c.nd * 2 * c.iwf * c.nkp_eom;
  k_add_siw<<<(int)std::min<size_t>(cdiv_u(n, 256), 4096), 256, 0, st>>>(c, sig, c.nkp_eom);
  cudaError_t e = ADGA_LAUNCH_CHECK();
  if (e == cudaSuccess && sig_loc) {
    k_sigma_loc<<<c.nd2 * 2 * c.iwf, 256, 0, st>>>(c, sig, sig_loc);
    e = ADGA_LAUNCH_CHECK();
  }
  if (e == cudaSuccess && gloc) {
    k_gloc<<<c.iwmax, 256, 0, st>>>(c, sig, gloc);
    e = ADGA_LAUNCH_CHECK();
  }
  if (e == cudaSuccess && n_dga_k) {
    k_occ<<<cdiv_u(c.nkp_eom, 128), 128, 0, st>>>(c, c.nkp_eom, keom, sig, n_dga_k);
    e = ADGA_LAUNCH_CHECK();
    if (e == cudaSuccess && n_dga) {
      k_ndga<<<c.nd, 256, 0, st>>>(c, n_dga_k, n_dga);
      e = ADGA_LAUNCH_CHECK();
    }
  }
  return e;
}

cudaError_t launch_nfock(const DevCtx &c, z64 *nfock, cudaStream_t st) {
  if (c.nd > PL_MAXND) return cudaErrorInvalidValue;
  k_occ<<<cdiv_u(c.nkp, 128), 128, 0, st>>>(c, c.nkp, nullptr, nullptr, nfock);
  return ADGA_LAUNCH_CHECK();
}
