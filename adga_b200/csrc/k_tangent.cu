// Tangent (forward-mode) propagation through the BSE of one batch: the
// derivative of X = (1+gamma^w) A^-1 along a parameter direction,
//     dX = (dB - X dA) A^-1,   d(A^-1) = -A^-1 dA A^-1,
// with A = 1 - blockdiag_nu(sw) F~, sw = chi0^q chi0_loc^-1 - 1 (src/main.F90:674-737):
//     dA = -blockdiag(dchi0^q chi0_loc^-1) F~ - blockdiag(sw) dF~
//     -X dA = XS F~ + XD dF~,   XS = X blockdiag(dchi0 chi0_loc^-1), XD = X blockdiag(sw)
// k_tan_rhs forms r = dB + XS F~ + XD dF~ for one channel in FP64 (the same
// cp.async GEMM mainloop as the refinement residual); the solve r A^-1 reuses
// the batch's LU factors.  k_gamq_tan forms the tangent of gamma^q_d
// (the nu-block row sums of sw F~_d, src/main.F90:700).
#include "ctx.cuh"
#include "zgemm.cuh"
#include <algorithm>

using namespace zg;

__global__ void __launch_bounds__(NT)
k_tan_rhs(int N, int R, int npts, int ch, const z64 *__restrict__ XS, const z64 *__restrict__ Frow,
          const z64 *__restrict__ XD, const z64 *__restrict__ Fdot, const z64 *__restrict__ dB, z64 *out) {
  extern __shared__ __align__(16) z64 zg_smem[];
  z64 *As = zg_smem, *Bs = zg_smem + STAGES * BK * BM;
  const int t = threadIdx.x, tx = t & 15, ty = t >> 4;
  const int rows = npts * R;
  const int r0 = blockIdx.y * BM, c0 = blockIdx.x * BN;
  const size_t per = (size_t)R * N;
  z64 acc[TM][TN], acc2[TM][TN];
  auto la_of = [&](const z64 *A) {
    return [=](int r, int k) -> const z64 * {
      const int row = r0 + r;
      if (row >= rows || k >= N) return nullptr;
      const int p = row / R, i1 = row % R;
      return A + (size_t)(2 * p + ch) * per + (size_t)i1 * N + k;
    };
  };
  auto lb_of = [&](const z64 *B) {
    return [=](int k, int c) -> const z64 * {
      const int cl = c0 + c;
      return (k < N && cl < N) ? B + (size_t)k * N + cl : nullptr;
    };
  };
#pragma unroll
  for (int i = 0; i < TM; ++i)
#pragma unroll
    for (int j = 0; j < TN; ++j) acc[i][j] = acc2[i][j] = make_double2(0.0, 0.0);
  if (XS) mainloop<true, true>(acc, As, Bs, N, la_of(XS), lb_of(Frow), Frow);
  if (XD && Fdot) {
    __syncthreads();
    mainloop<true, true>(acc2, As, Bs, N, la_of(XD), lb_of(Fdot), Fdot);
  }
#pragma unroll
  for (int i = 0; i < TM; ++i) {
    const int row = r0 + tx + 16 * i;
    if (row >= rows) continue;
    const int p = row / R, i1 = row % R;
    const size_t m = (size_t)(2 * p + ch);
#pragma unroll
    for (int j = 0; j < TN; ++j) {
      const int cl = c0 + ty + 16 * j;
      if (cl >= N) continue;
      z64 v = cadd(acc[i][j], acc2[i][j]);
      if (dB) v = cadd(v, dB[i1 + (size_t)cl * R]);
      out[m * per + (size_t)i1 * N + cl] = v;
    }
  }
}

cudaError_t launch_tan_rhs(const DevCtx &c, int npts, int ch, const z64 *XS, const z64 *Frow, const z64 *XD,
                           const z64 *Fdot, const z64 *dB, z64 *out, cudaStream_t st) {
  smem_limit(k_tan_rhs, SMEM_BYTES);
  dim3 g(cdiv_u(c.N, BN), cdiv_u((size_t)npts * c.R, BM));
  k_tan_rhs<<<g, NT, SMEM_BYTES, st>>>(c.N, c.R, npts, ch, XS, Frow, XD, Fdot, dB, out);
  return ADGA_LAUNCH_CHECK();
}

// dgamma^q_d(p)(i1, cc) = sum_nu sum_i3 [dsw(i1,i3) F~_d(i3 + nu nd2, cc) + sw(i1,i3) dF~_d(i3 + nu nd2, cc)]
template <int ND2>
__global__ void __launch_bounds__(128)
k_gamq_tan(DevCtx c, const z64 *__restrict__ chi0q, const z64 *__restrict__ dchi0q, const z64 *__restrict__ c0inv,
           const z64 *__restrict__ Frow_d, const z64 *__restrict__ Fdot_d, z64 *dgq) {
  __shared__ z64 sw[ND2 * ND2], dsw[ND2 * ND2];
  const int N = c.N, cc = blockIdx.x * blockDim.x + threadIdx.x, p = blockIdx.y;
  const z64 *c0 = chi0q + (size_t)p * ND2 * ND2 * 2 * c.iwf;
  const z64 *d0 = dchi0q ? dchi0q + (size_t)p * ND2 * ND2 * 2 * c.iwf : nullptr;
  z64 acc[ND2];
#pragma unroll
  for (int a = 0; a < ND2; ++a) acc[a] = make_double2(0.0, 0.0);
  for (int dum = 0; dum < 2 * c.iwf; ++dum) {
    __syncthreads();
    for (int e = threadIdx.x; e < ND2 * ND2; e += blockDim.x) {
      const int i1 = e % ND2, i3 = e / ND2;
      const z64 ci = c0inv[dum * ND2 + i3];
      z64 v = cmul(c0[(size_t)dum * ND2 * ND2 + e], ci);
      if (i1 == i3) v.x -= 1.0;
      sw[e] = v;
      dsw[e] = d0 ? cmul(d0[(size_t)dum * ND2 * ND2 + e], ci) : make_double2(0.0, 0.0);
    }
    __syncthreads();
    if (cc < N) {
      z64 f[ND2], fd[ND2];
#pragma unroll
      for (int i3 = 0; i3 < ND2; ++i3) {
        f[i3] = d0 ? Frow_d[(size_t)(i3 + dum * ND2) * N + cc] : make_double2(0.0, 0.0);
        fd[i3] = Fdot_d ? Fdot_d[(size_t)(i3 + dum * ND2) * N + cc] : make_double2(0.0, 0.0);
      }
#pragma unroll
      for (int i1 = 0; i1 < ND2; ++i1)
#pragma unroll
        for (int i3 = 0; i3 < ND2; ++i3) {
          cfma(acc[i1], dsw[i1 + i3 * ND2], f[i3]);
          cfma(acc[i1], sw[i1 + i3 * ND2], fd[i3]);
        }
    }
  }
  if (cc < N)
#pragma unroll
    for (int i1 = 0; i1 < ND2; ++i1) dgq[(size_t)p * ND2 * N + i1 + (size_t)cc * ND2] = acc[i1];
}

cudaError_t launch_gamq_tan(const DevCtx &c, int npts, const z64 *chi0q, const z64 *dchi0q, const z64 *c0inv,
                            const z64 *Frow_d, const z64 *Fdot_d, z64 *dgq, cudaStream_t st) {
  if (npts <= 0) return cudaSuccess;
  dim3 grid(cdiv_u(c.N, 128), npts);
#define GQT(NDD) k_gamq_tan<NDD><<<grid, 128, 0, st>>>(c, chi0q, dchi0q, c0inv, Frow_d, Fdot_d, dgq)
  switch (c.nd2) {
    case 1: GQT(1); break;
    case 4: GQT(4); break;
    case 9: GQT(9); break;
    case 16: GQT(16); break;
    case 25: GQT(25); break;
    default: return cudaErrorInvalidValue;
  }
#undef GQT
  return ADGA_LAUNCH_CHECK();
}

__global__ void k_zadd(size_t n, const z64 *__restrict__ x, z64 *__restrict__ y) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    y[i] = cadd(y[i], x[i]);
}

cudaError_t launch_zadd(size_t n, const z64 *x, z64 *y, cudaStream_t st) {
  if (!n) return cudaSuccess;
  k_zadd<<<(int)std::min<size_t>(cdiv_u(n, 256), 4096), 256, 0, st>>>(n, x, y);
  return ADGA_LAUNCH_CHECK();
}
