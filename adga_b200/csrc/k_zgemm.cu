// Complex FP64 GEMMs on the CUDA cores built on zgemm.cuh:
//   * k_trail_z64  -- the FP64 LU trailing update A22 -= L21 U12 (batched);
//   * k_resid_z64  -- the refinement residual r = B - X + (X D) F~ of the
//                     mixed path (rows = points x ndim2, K = N, F~ shared).
#include "ctx.cuh"
#include "lu.cuh"
#include "zgemm.cuh"

using namespace zg;

__global__ void __launch_bounds__(NT)
k_trail_z64(z64 *M, size_t strideM, int N, int ncols, int J, int jb) {
  extern __shared__ __align__(16) z64 zg_smem[];
  z64 *As = zg_smem, *Bs = zg_smem + STAGES * BK * BM;
  const int t = threadIdx.x, tx = t & 15, ty = t >> 4;
  z64 *A = M + (size_t)blockIdx.z * strideM;
  const int r0 = J + jb + blockIdx.y * BM, c0 = J + jb + blockIdx.x * BN;
  auto la = [&](int r, int k) -> const z64 * {
    const int rr = r0 + r;
    return (rr < N && k < jb) ? A + rr + (size_t)(J + k) * N : nullptr;
  };
  auto lb = [&](int k, int c) -> const z64 * {
    const int cc = c0 + c;
    return (k < jb && cc < ncols) ? A + (J + k) + (size_t)cc * N : nullptr;
  };
  z64 acc[TM][TN];
  mainloop<false, false>(acc, As, Bs, jb, la, lb, A);
  z64 cv[TM][TN];
#pragma unroll
  for (int j = 0; j < TN; ++j)
#pragma unroll
    for (int i = 0; i < TM; ++i) {
      const int r = r0 + tx + 16 * i, c = c0 + ty + 16 * j;
      cv[i][j] = (r < N && c < ncols) ? A[r + (size_t)c * N] : make_double2(0.0, 0.0);
    }
#pragma unroll
  for (int j = 0; j < TN; ++j)
#pragma unroll
    for (int i = 0; i < TM; ++i) {
      const int r = r0 + tx + 16 * i, c = c0 + ty + 16 * j;
      if (r < N && c < ncols) A[r + (size_t)c * N] = csub(cv[i][j], acc[i][j]);
    }
}

cudaError_t lu_trail_z64(z64 *M, const LUBatch &lb, int J, int jb, cudaStream_t st) {
  const int m = lb.N - J - jb, n = lb.ncols - J - jb;
  if (m <= 0 || n <= 0) return cudaSuccess;
  smem_limit(k_trail_z64, SMEM_BYTES);
  dim3 grid(cdiv_u(n, BN), cdiv_u(m, BM), lb.batch);
  k_trail_z64<<<grid, NT, SMEM_BYTES, st>>>(M, lb.strideM, lb.N, lb.ncols, J, jb);
  return ADGA_LAUNCH_CHECK();
}

// rows (p, i1) of channel ch, columns c:
//   V(p,i1,c) = fp32( opg(i1,c) - X(p,i1,c) + sum_m XD(p,i1,m) F~(m,c) )
__global__ void __launch_bounds__(NT)
k_resid_z64(int N, int R, int npts, int ch, const z64 *__restrict__ XD, const z64 *__restrict__ X,
            const z64 *__restrict__ Frow, const z64 *__restrict__ opg, z32 *V, const z64 *__restrict__ extra,
            unsigned long long *rnorm, const z64 *__restrict__ Bpt) {
  extern __shared__ __align__(16) z64 zg_smem[];
  z64 *As = zg_smem, *Bs = zg_smem + STAGES * BK * BM;
  const int t = threadIdx.x, tx = t & 15, ty = t >> 4;
  const int rows = npts * R;
  const int r0 = blockIdx.y * BM, c0 = blockIdx.x * BN;
  const size_t per = (size_t)R * N;
  auto la = [&](int r, int k) -> const z64 * {
    const int row = r0 + r;
    if (row >= rows || k >= N) return nullptr;
    const int p = row / R, i1 = row % R;
    return XD + (size_t)(2 * p + ch) * per + (size_t)i1 * N + k;
  };
  auto lb = [&](int k, int c) -> const z64 * {
    const int cl = c0 + c;
    return (k < N && cl < N) ? Frow + (size_t)k * N + cl : nullptr;
  };
  z64 acc[TM][TN];
  mainloop<true, true>(acc, As, Bs, N, la, lb, Frow);
#pragma unroll
  for (int i = 0; i < TM; ++i) {
    const int row = r0 + tx + 16 * i;
    const int p = row / R, i1 = row % R;
    const size_t m = (size_t)(2 * p + ch);
    double rmax = 0.0;
#pragma unroll
    for (int j = 0; j < TN; ++j) {
      const int cl = c0 + ty + 16 * j;
      if (row >= rows || cl >= N) continue;
      // right-hand side: (1+gamma^w) shared by the slice, or per point (tangent solves)
      const z64 b = Bpt ? Bpt[m * per + (size_t)i1 * N + cl] : opg[i1 + (size_t)cl * R];
      const z64 x = X[m * per + (size_t)i1 * N + cl];
      z64 r = make_double2(b.x - x.x + acc[i][j].x, b.y - x.y + acc[i][j].y);
      if (extra) r = cadd(r, extra[(size_t)p * per + (size_t)i1 * N + cl]);   // V(q) term (density)
      V[m * per + (size_t)i1 * N + cl] = to32(r);
      rmax = fmax(rmax, fabs(r.x) + fabs(r.y));
    }
    // max |re| + |im| of the FP64 residual per matrix (lanes t and t + 16 share their rows)
    rmax = fmax(rmax, __shfl_xor_sync(0xffffffffu, rmax, 16));
    if (rnorm && ty % 2 == 0 && row < rows && rmax > 0.0)
      atomicMax(rnorm + (size_t)(2 * p + ch), (unsigned long long)__double_as_longlong(rmax));
  }
}

cudaError_t launch_resid_z64(const DevCtx &c, int npts, const z64 *XD, const z64 *X,
                             const z64 *Frow_d, const z64 *Frow_m, const z64 *opg_d,
                             const z64 *opg_m, z32 *V, const z64 *extra_d, unsigned long long *rnorm,
                             const z64 *Bpt, cudaStream_t st) {
  smem_limit(k_resid_z64, SMEM_BYTES);
  dim3 g(cdiv_u(c.N, BN), cdiv_u((size_t)npts * c.R, BM));
  k_resid_z64<<<g, NT, SMEM_BYTES, st>>>(c.N, c.R, npts, 0, XD, X, Frow_d, opg_d, V, extra_d, rnorm, Bpt);
  cudaError_t e = ADGA_LAUNCH_CHECK();
  if (e != cudaSuccess) return e;
  k_resid_z64<<<g, NT, SMEM_BYTES, st>>>(c.N, c.R, npts, 1, XD, X, Frow_m, opg_m, V, nullptr, rnorm, Bpt);
  return ADGA_LAUNCH_CHECK();
}
