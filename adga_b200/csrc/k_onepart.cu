// One-particle and per-omega local kernels of the ladder hot path.
//
//  * G(k, nu) table      -- the Green's functions accumulate_chi0 and get_gkiw
//                           rebuild on the fly (src/one_particle_quant_module.f90:81-104,240-271)
//  * k - q index         -- index_kq (src/kq_tools.f90:59-108)
//  * local block         -- src/main.F90:506-627 (chi0_loc, F~, gamma^w, 1+gamma^w)
//  * local EOM parts     -- calc_eom_static / calc_eom_dmft (src/eom_module.f90:39-161)
#include "ctx.cuh"
#include "ginv.cuh"

#define MAXND GINV_MAXND

__global__ void k_gtable(DevCtx c, z64 *gtab) {
  size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  size_t total = (size_t)c.nkp * c.nnu;
  if (idx >= total) return;
  int k = (int)(idx % c.nkp);
  int nu = (int)(idx / c.nkp) + c.nu_lo;
  int nd = c.nd;
  z64 a[MAXND * MAXND];
  const z64 *h = c.hk + (size_t)k * c.nd2;
  for (int i = 0; i < nd * nd; ++i) a[i] = cneg(h[i]);
  double w = c.iw[nu + c.iwmax];
  for (int i = 0; i < nd; ++i) {
    z64 d = make_double2(c.mu, w);               // ci*iw + mu
    d = csub(d, h[i + i * nd]);                   // - hk(i,i)
    d = csub(d, c.dc[2 * i]);                     // - dc(1,i)
    d = csub(d, c.siw[(nu + c.iwmax) + i * 2 * c.iwmax]);  // - siw(nu,i)
    a[i + i * nd] = d;
  }
  ginv_small(nd, a);
  z64 *o = gtab + idx * c.nd2;
  for (int i = 0; i < nd * nd; ++i) o[i] = a[i];
}

// tangent of the G table for a direction dH(k): dG = G dH G (the self-energy,
// mu and dc are held fixed)
__global__ void k_gtable_dot(DevCtx c, const z64 *__restrict__ dhk, z64 *__restrict__ gdot) {
  size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  size_t total = (size_t)c.nkp * c.nnu;
  if (idx >= total) return;
  const int k = (int)(idx % c.nkp), nd = c.nd;
  const z64 *g = c.gtab + idx * c.nd2, *dh = dhk + (size_t)k * c.nd2;
  z64 t[MAXND * MAXND];
  for (int i = 0; i < nd; ++i)
    for (int j = 0; j < nd; ++j) {
      z64 s = czero<z64>();
      for (int m = 0; m < nd; ++m) cfma(s, g[i + m * nd], dh[m + j * nd]);
      t[i + j * nd] = s;
    }
  for (int i = 0; i < nd; ++i)
    for (int j = 0; j < nd; ++j) {
      z64 s = czero<z64>();
      for (int m = 0; m < nd; ++m) cfma(s, t[i + m * nd], g[m + j * nd]);
      gdot[idx * c.nd2 + i + j * nd] = s;
    }
}

cudaError_t launch_gtable_dot(const DevCtx &c, const z64 *dhk, z64 *gdot, cudaStream_t st) {
  size_t total = (size_t)c.nkp * c.nnu;
  k_gtable_dot<<<cdiv_u(total, 128), 128, 0, st>>>(c, dhk, gdot);
  return ADGA_LAUNCH_CHECK();
}

cudaError_t launch_gtable(const DevCtx &c, z64 *gtab, cudaStream_t st) {
  size_t total = (size_t)c.nkp * c.nnu;
  k_gtable<<<cdiv_u(total, 128), 128, 0, st>>>(c, gtab);
  return ADGA_LAUNCH_CHECK();
}

// ---------------------------------------------------------------------------
// k - q index (src/kq_tools.f90:96-108), ind(k, q) column-major.
// ---------------------------------------------------------------------------
__global__ void k_kq_index(int nx, int ny, int nz, const int *k_sel, int nk_sel,
                           const int *q_data, int nqp, int one_based, int *ind) {
  size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (idx >= (size_t)nk_sel * nqp) return;
  int kk = (int)(idx % nk_sel), jq = (int)(idx / nk_sel);
  int ik = k_sel ? k_sel[kk] : kk + 1;     // 1-based
  int iq = q_data[jq];                     // 1-based
  int iz = (ik - 1) % nz, iy = ((ik - 1) / nz) % ny, ix = (ik - 1) / (ny * nz);
  int lz = (iq - 1) % nz, ly = ((iq - 1) / nz) % ny, lx = (iq - 1) / (ny * nz);
  int r = 1 + (nz + iz - lz) % nz + ((ny + iy - ly) % ny) * nz + ((nx + ix - lx) % nx) * ny * nz;
  ind[idx] = one_based ? r : r - 1;
}

cudaError_t launch_kq_index(int nkpx, int nkpy, int nkpz, const int *k_sel, int nk_sel,
                            const int *q_data, int nqp, int one_based, int *ind, cudaStream_t st) {
  size_t total = (size_t)nk_sel * nqp;
  if (total == 0) return cudaSuccess;
  k_kq_index<<<cdiv_u(total, 256), 256, 0, st>>>(nkpx, nkpy, nkpz, k_sel, nk_sel, q_data, nqp,
                                                 one_based, ind);
  return ADGA_LAUNCH_CHECK();
}

// ---------------------------------------------------------------------------
// Local block of one omega (src/main.F90:508-521): diagonals of
// chi0_loc^-1 and chi0_loc in the big index i2 + dum*nd2, and
// bubble_loc_tmp = sum_{iwstart..iwstop} chi0_loc / beta^2.
// ---------------------------------------------------------------------------
__device__ __forceinline__ z64 giw_at(const DevCtx &c, int n, int i) {
  return c.giw[(n + c.iwmax) + i * 2 * c.iwmax];
}

__global__ void k_local_diag(DevCtx c, int iwb, z64 *c0inv, z64 *c0w, z64 *bubloc_tmp) {
  int nd = c.nd, nd2 = c.nd2;
  int tid = blockIdx.x * blockDim.x + threadIdx.x;
  int nsmall = 2 * c.iwf * nd2;
  if (tid < nsmall) {
    int dum = tid / nd2, i2 = tid % nd2;
    int i = i2 / nd, j = i2 % nd;          // i2 = {j,i}: j fastest
    int iwf = dum - c.iwf;
    z64 gi = giw_at(c, iwf, i), gj = giw_at(c, iwf - iwb, j);
    // -1/(beta*g_i*g_j)  (get_chi0_loc_inv)
    z64 t = cmul(cscale(gi, c.beta), gj);
    c0inv[tid] = cneg(crcp(t));
    // -beta*g_i*g_j      (get_chi0_loc)
    c0w[tid] = cmul(cscale(gi, -c.beta), gj);
  } else if (tid < nsmall + nd2) {
    int i2 = tid - nsmall;
    int i = i2 / nd, j = i2 % nd;
    z64 s = czero<z64>();
    for (int iwf = c.iwstart; iwf <= c.iwstop; ++iwf)
      s = cadd(s, cmul(cscale(giw_at(c, iwf, i), -c.beta), giw_at(c, iwf - iwb, j)));
    double b2 = c.beta * c.beta;
    // bubble_loc_tmp is diagonal in the compound index (zeroed by the launcher)
    bubloc_tmp[i2 + i2 * nd2] = make_double2(s.x / b2, s.y / b2);
  }
}

cudaError_t launch_local_diag(const DevCtx &c, int iwb, z64 *c0inv, z64 *c0w, z64 *bubloc_tmp,
                              cudaStream_t st) {
  int n = 2 * c.iwf * c.nd2 + c.nd2;
  cudaError_t e = cudaMemsetAsync(bubloc_tmp, 0, sizeof(z64) * c.nd2 * c.nd2, st);
  if (e != cudaSuccess) return e;
  k_local_diag<<<cdiv_u(n, 128), 128, 0, st>>>(c, iwb, c0inv, c0w, bubloc_tmp);
  return ADGA_LAUNCH_CHECK();
}

// F~ = sym(chi_loc) * diag(chi0_loc^-1) - 1 (src/main.F90:529-553), written
// row-major: Frow[r*N + c] = F~(r, c).  chi_loc is column-major.
__global__ void k_local_F(int N, const z64 *chi, const z64 *c0inv, z64 *Frow, int minus_one) {
  __shared__ z64 A[32][33];   // A[cc][rr] = chi(r0+rr, c0+cc)
  __shared__ z64 B[32][33];   // B[rr][cc] = chi(c0+cc, r0+rr)
  int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
  int tx = threadIdx.x, ty = threadIdx.y;   // 32 x 8
  for (int k = ty; k < 32; k += 8) {
    int r = r0 + tx, cc = c0 + k;
    A[k][tx] = (r < N && cc < N) ? chi[r + (size_t)cc * N] : czero<z64>();
    int rr = r0 + k, c2 = c0 + tx;
    B[k][tx] = (rr < N && c2 < N) ? chi[c2 + (size_t)rr * N] : czero<z64>();
  }
  __syncthreads();
  for (int k = ty; k < 32; k += 8) {
    int r = r0 + k, cc = c0 + tx;
    if (r < N && cc < N) {
      z64 a = A[tx][k], b = B[k][tx];
      z64 s = (r == cc) ? a : make_double2(0.5 * (a.x + b.x), 0.5 * (a.y + b.y));
      z64 v = cmul(s, c0inv[cc]);
      if (r == cc && minus_one) v.x -= 1.0;
      Frow[(size_t)r * N + cc] = v;
    }
  }
}

cudaError_t launch_local_F(const DevCtx &c, const z64 *chi_loc, const z64 *c0inv, z64 *Frow,
                           cudaStream_t st, bool minus_one) {
  dim3 grid(cdiv_u(c.N, 32), cdiv_u(c.N, 32));
  k_local_F<<<grid, dim3(32, 8), 0, st>>>(c.N, chi_loc, c0inv, Frow, minus_one ? 1 : 0);
  return ADGA_LAUNCH_CHECK();
}

// gamma^w(i1, :) = sum_dum F~(i1 + dum*nd2, :) and 1 + gamma^w
// (src/main.F90:564-570, 617-625); column-major (nd2, N).
__global__ void k_local_gamma(int N, int nd2, int n2iwf, const z64 *Frow, z64 *gam, z64 *opg) {
  size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (idx >= (size_t)nd2 * N) return;
  int cc = (int)(idx % N), i1 = (int)(idx / N);
  z64 s = czero<z64>();
  for (int dum = 0; dum < n2iwf; ++dum) s = cadd(s, Frow[(size_t)(i1 + dum * nd2) * N + cc]);
  gam[i1 + (size_t)cc * nd2] = s;
  if (cc % nd2 == i1) s.x += 1.0;
  opg[i1 + (size_t)cc * nd2] = s;
}

cudaError_t launch_local_gamma(const DevCtx &c, const z64 *Frow, z64 *gam, z64 *opg, cudaStream_t st) {
  size_t total = (size_t)c.nd2 * c.N;
  k_local_gamma<<<cdiv_u(total, 256), 256, 0, st>>>(c.N, c.nd2, 2 * c.iwf, Frow, gam, opg);
  return ADGA_LAUNCH_CHECK();
}

// chi_loc(w) += calc_chi_qw(gamma^w, chi0w) for both channels
// (src/main.F90:573-577) and bubble_loc(w) += bubble_loc_tmp (:521).
__global__ void k_chi_loc_update(DevCtx c, const z64 *gd, const z64 *gm, const z64 *c0w,
                                 const z64 *bub_tmp, z64 *cld, z64 *clm, z64 *bub_loc) {
  int nd2 = c.nd2;
  int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= nd2 * nd2) return;
  int i1 = idx % nd2, i2 = idx / nd2;
  z64 sd = czero<z64>(), sm = czero<z64>();
  for (int dum = 0; dum < 2 * c.iwf; ++dum) {
    z64 w = c0w[dum * nd2 + i2];
    size_t col = (size_t)(i2 + dum * nd2) * nd2;
    cfma(sd, gd[i1 + col], w);
    cfma(sm, gm[i1 + col], w);
  }
  double b2 = c.beta * c.beta;
  if (cld) {   // null with an external chi_loc: only the bubble accumulates (src/main.F90:573)
    cld[idx] = cadd(cld[idx], make_double2(sd.x / b2, sd.y / b2));
    clm[idx] = cadd(clm[idx], make_double2(sm.x / b2, sm.y / b2));
  }
  bub_loc[idx] = cadd(bub_loc[idx], bub_tmp[idx]);
}

cudaError_t launch_chi_loc_update(const DevCtx &c, const z64 *gam_d, const z64 *gam_m,
                                  const z64 *c0w, const z64 *bubloc_tmp, z64 *chi_loc_d,
                                  z64 *chi_loc_m, z64 *bubble_loc, cudaStream_t st) {
  int n = c.nd2 * c.nd2;
  k_chi_loc_update<<<cdiv_u(n, 128), 128, 0, st>>>(c, gam_d, gam_m, c0w, bubloc_tmp, chi_loc_d,
                                                   chi_loc_m, bubble_loc);
  return ADGA_LAUNCH_CHECK();
}

// ---------------------------------------------------------------------------
// calc_eom_static, local Hartree term (src/eom_module.f90:52-70):
// sigma_dmft(i,i,:) += sum_j (2 u({ii},{jj}) - u({ji},{ji})) n_dmft(j)
// ---------------------------------------------------------------------------
__global__ void k_eom_static(DevCtx c, z64 *sig) {
  int nd = c.nd, nd2 = c.nd2;
  int i = threadIdx.x;
  if (i >= nd) return;
  z64 t = czero<z64>();
  int i1 = i * nd + i;
  for (int j = 0; j < nd; ++j) {
    int i2 = j * nd + j, i3 = i * nd + j;
    z64 a = c.u[i1 + i2 * nd2], b = c.u[i3 + i3 * nd2];
    z64 f = make_double2(2.0 * a.x - b.x, 2.0 * a.y - b.y);
    cfma(t, f, c.ndmft[j]);
  }
  for (int w = 0; w < 2 * c.iwf; ++w) {
    size_t o = i + i * nd + (size_t)w * nd2;
    sig[o] = cadd(sig[o], t);
  }
}

cudaError_t launch_eom_static(const DevCtx &c, z64 *sigma_dmft, cudaStream_t st) {
  k_eom_static<<<1, 32, 0, st>>>(c, sigma_dmft);
  return ADGA_LAUNCH_CHECK();
}

// calc_eom_dmft (src/eom_module.f90:138-158): m_tot = -(1/beta) u . gamma^w_d;
// sigma(i,l,nu) += sum_k m_tot({k,i},{k,l,nu}) giw(nu-w, k) for nu >= 0.
__global__ void k_eom_dmft(DevCtx c, int iwb, const z64 *gd, z64 *sig) {
  int nd = c.nd, nd2 = c.nd2;
  int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= nd2 * c.iwf) return;
  int i = idx % nd, l = (idx / nd) % nd, nu = idx / nd2;
  size_t o = i + l * nd + (size_t)(nu + c.iwf) * nd2;
  z64 s = sig[o];
  for (int k = 0; k < nd; ++k) {
    int i1 = i * nd + k;                               // {k,i}
    size_t col = (size_t)(nu + c.iwf) * nd2 + l * nd + k;   // {k,l,nu}
    z64 m = czero<z64>();
    for (int i3 = 0; i3 < nd2; ++i3) cfma(m, c.u[i1 + i3 * nd2], gd[i3 + col * nd2]);
    m = cscale(m, -1.0 / c.beta);
    cfma(s, m, giw_at(c, nu - iwb, k));
  }
  sig[o] = s;
}

// Sigma(:,:,-nu-1) = Sigma(:,:,nu)^dagger for nu in [0, iwf) at each of nk
// k-points (src/eom_module.f90:157,228).
__global__ void k_mirror_sigma(int nd, int iwf, int nk, z64 *sig) {
  size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  size_t nd2 = (size_t)nd * nd;
  if (idx >= nd2 * iwf * nk) return;
  int i = idx % nd, l = (idx / nd) % nd;
  int nu = (int)((idx / nd2) % iwf);
  size_t k = idx / (nd2 * iwf);
  size_t base = k * nd2 * 2 * iwf;
  z64 v = sig[base + l + i * nd + (size_t)(nu + iwf) * nd2];
  sig[base + i + l * nd + (size_t)(iwf - 1 - nu) * nd2] = cconj(v);
}

cudaError_t launch_eom_dmft(const DevCtx &c, int iwb, const z64 *gam_d, z64 *sigma_dmft,
                            cudaStream_t st) {
  int n = c.nd2 * c.iwf;
  k_eom_dmft<<<cdiv_u(n, 64), 64, 0, st>>>(c, iwb, gam_d, sigma_dmft);
  cudaError_t e = ADGA_LAUNCH_CHECK();
  if (e != cudaSuccess) return e;
  return launch_mirror_sigma(c, sigma_dmft, 1, st);
}

cudaError_t launch_mirror_sigma(const DevCtx &c, z64 *sigma, int nk, cudaStream_t st) {
  size_t total = (size_t)c.nd2 * c.iwf * nk;
  if (!total) return cudaSuccess;
  k_mirror_sigma<<<cdiv_u(total, 256), 256, 0, st>>>(c.nd, c.iwf, nk, sigma);
  return ADGA_LAUNCH_CHECK();
}

// calc_chi_qw (src/susc_module.f90:34-56) on device buffers:
// chi_qw += beta^-2 sum_{dum,i3} interm3(:, i3+dum*nd2) * chi0_sum(i3, :, dum)
__global__ void k_calc_chi_qw(DevCtx c, z64 *chi, const z64 *im3, const z64 *c0s) {
  int nd2 = c.nd2;
  int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= nd2 * nd2) return;
  int i1 = idx % nd2, i2 = idx / nd2;
  z64 s = czero<z64>();
  for (int dum = 0; dum < 2 * c.iwf; ++dum)
    for (int i3 = 0; i3 < nd2; ++i3)
      cfma(s, im3[i1 + (size_t)(i3 + dum * nd2) * nd2],
           c0s[i3 + i2 * nd2 + (size_t)dum * nd2 * nd2]);
  double b2 = c.beta * c.beta;
  chi[idx] = cadd(chi[idx], make_double2(s.x / b2, s.y / b2));
}

cudaError_t launch_calc_chi_qw(const DevCtx &c, z64 *chi_qw, const z64 *interm3,
                               const z64 *chi0_sum, cudaStream_t st) {
  int n = c.nd2 * c.nd2;
  k_calc_chi_qw<<<cdiv_u(n, 64), 64, 0, st>>>(c, chi_qw, interm3, chi0_sum);
  return ADGA_LAUNCH_CHECK();
}
