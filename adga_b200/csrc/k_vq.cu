// Non-local interaction V(q) (do_vq): the parts of the ladder that V(q)
// enters besides the BSE build and m_tot (k_bse.cu).
//   read_vq's index map   v(i1 = i nd + k, i2 = l nd + j, q) = vq(i, j, k, l, q)
//                         (src/interaction_module.f90:107-119)
//   calc_eom_static       non-local Hartree 2 v(q=0) n_dmft and Fock
//                         -v(q)/nqp n_fock(k-q) into sigma_hf (src/eom_module.f90:70-108)
//   mixed refinement      the density-channel residual term X blockdiag(S_nu) (1+gamma^w_d),
//                         S_nu = 2 beta^-2 chi0^q(nu) v(q), i.e. Y (1+gamma^w_d) with
//                         Y = 2 beta^-2 sum_nu X_nu chi0^q(nu) v(q)
#include "ctx.cuh"

__global__ void k_vq_permute(int nd, int nqp, const z64 *__restrict__ raw, z64 *__restrict__ v) {
  const int nd2 = nd * nd;
  const size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (idx >= (size_t)nd2 * nd2 * nqp) return;
  const int i1 = (int)(idx % nd2), i2 = (int)((idx / nd2) % nd2);
  const size_t q = idx / ((size_t)nd2 * nd2);
  const int i = i1 / nd, k = i1 % nd, l = i2 / nd, j = i2 % nd;
  v[idx] = raw[(size_t)i + nd * ((size_t)j + nd * ((size_t)k + nd * ((size_t)l + nd * q)))];
}

cudaError_t launch_vq_permute(int nd, int nqp, const z64 *raw, z64 *v, cudaStream_t st) {
  const size_t total = (size_t)nd * nd * nd * nd * nqp;
  k_vq_permute<<<cdiv_u(total, 256), 256, 0, st>>>(nd, nqp, raw, v);
  return ADGA_LAUNCH_CHECK();
}

// sigma_hf(i, l, ik) for the points of one batch at omega = 0, in point order
__global__ void k_eom_static_vq(DevCtx c, const int *__restrict__ qidx, int npts, z64 *sigma_hf) {
  const int nd = c.nd, nd2 = c.nd2;
  const size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (idx >= (size_t)nd2 * c.nkp_eom) return;
  const int i = (int)(idx % nd), l = (int)((idx / nd) % nd);
  const size_t ik = idx / nd2;
  z64 s = sigma_hf[idx];
  for (int p = 0; p < npts; ++p) {
    const int q = qidx[p];
    const z64 *v = c.vq + (size_t)q * nd2 * nd2;
    if (q == 0 && i == l)                     // q = 0: non-local Hartree 2 v(q=0) n_dmft
      for (int j = 0; j < nd; ++j) {
        const z64 t = cmul(v[(i * nd + i) + (size_t)(j * nd + j) * nd2], c.ndmft[j]);
        s = cadd(s, make_double2(2.0 * t.x, 2.0 * t.y));
      }
    const int ikq = c.kqe[ik + (size_t)q * c.nkp_eom];
    for (int j = 0; j < nd; ++j)               // Fock: -v({ki},{jl})/nqp n_fock(k-q, j, k)
      for (int k = 0; k < nd; ++k) {
        const z64 vv = v[(i * nd + k) + (size_t)(l * nd + j) * nd2];
        const z64 a = make_double2(vv.x / c.nqp, vv.y / c.nqp);
        s = csub(s, cmul(a, c.nfock[(size_t)ikq + (size_t)c.nkp * (j + (size_t)nd * k)]));
      }
  }
  sigma_hf[idx] = s;
}

cudaError_t launch_eom_static_vq(const DevCtx &c, const int *qidx, int npts, z64 *sigma_hf, cudaStream_t st) {
  const size_t total = (size_t)c.nd2 * c.nkp_eom;
  k_eom_static_vq<<<cdiv_u(total, 128), 128, 0, st>>>(c, qidx, npts, sigma_hf);
  return ADGA_LAUNCH_CHECK();
}

// extra(p, i1, c) = sum_j Y_p(i1, j) (1+gamma^w_d)(j, c) for the density channel
// (matrix 2p of X); one block per point
__global__ void __launch_bounds__(256)
k_vq_resid_extra(DevCtx c, const int *__restrict__ qidx, const z64 *__restrict__ X, const z64 *__restrict__ chi0q,
                 const z64 *__restrict__ opg_d, z64 *__restrict__ extra) {
  extern __shared__ z64 sy[];                  // Z then Y, nd2 x nd2 each
  const int p = blockIdx.x, nd2 = c.nd2, N = c.N, t = threadIdx.x;
  const size_t per = (size_t)nd2 * N;
  const z64 *x = X + (size_t)(2 * p) * per;
  const z64 *cq = chi0q + (size_t)p * nd2 * nd2 * 2 * c.iwf;
  z64 *Z = sy, *Y = sy + nd2 * nd2;
  // Z(i1, n) = sum_nu sum_m X(i1, nu nd2 + m) chi0q(m, n, nu)
  for (int e = t; e < nd2 * nd2; e += blockDim.x) {
    const int i1 = e % nd2, n = e / nd2;
    z64 s = make_double2(0.0, 0.0);
    for (int nu = 0; nu < 2 * c.iwf; ++nu)
      for (int m = 0; m < nd2; ++m)
        cfma(s, x[(size_t)i1 * N + nu * nd2 + m], cq[m + (size_t)n * nd2 + (size_t)nu * nd2 * nd2]);
    Z[e] = s;
  }
  __syncthreads();
  const z64 *v = c.vq + (size_t)qidx[p] * nd2 * nd2;
  const double f = 2.0 / (c.beta * c.beta);
  for (int e = t; e < nd2 * nd2; e += blockDim.x) {
    const int i1 = e % nd2, j = e / nd2;
    z64 s = make_double2(0.0, 0.0);
    for (int n = 0; n < nd2; ++n) cfma(s, Z[i1 + n * nd2], v[n + (size_t)j * nd2]);
    Y[e] = make_double2(f * s.x, f * s.y);
  }
  __syncthreads();
  z64 *o = extra + (size_t)p * per;
  for (size_t e = t; e < per; e += blockDim.x) {
    const int i1 = (int)(e / N), col = (int)(e % N);
    z64 s = make_double2(0.0, 0.0);
    for (int j = 0; j < nd2; ++j) cfma(s, Y[i1 + j * nd2], opg_d[j + (size_t)col * nd2]);
    o[e] = s;
  }
}

cudaError_t launch_vq_resid_extra(const DevCtx &c, int npts, const int *qidx, const z64 *X, const z64 *chi0q,
                                  const z64 *opg_d, z64 *extra, cudaStream_t st) {
  if (npts <= 0) return cudaSuccess;
  k_vq_resid_extra<<<npts, 256, 2 * sizeof(z64) * c.nd2 * c.nd2, st>>>(c, qidx, X, chi0q, opg_d, extra);
  return ADGA_LAUNCH_CHECK();
}
