// FP64 iterative refinement of the mixed-precision BSE solve.
//
// The unknown is X = (1+gamma^w) A^-1 (ndim2 x N), solved from
// X A = B with A = 1 - D F~ (D = blockdiag_nu(chi0^q chi0_loc^-1 - 1)).
// The residual never needs A in FP64:
//     r = B - X A = B - X + (X D) F~ ,
// a (ndim2 x N) x (N x N) product per point with F~ shared by all q of one
// omega (L2-resident), computed here as one batched FP64 GEMM per channel.
// The correction d A = r is solved with the FP32 LU factors (forward with
// L and the pivots, backward with U), and X += d in FP64.
//
// Buffers follow the LU batch order m = 2*p + ch.  X (FP64) and the FP32
// right-hand sides V are N x R column-major per matrix, which is the same
// memory as X stored R x N row-major.
#include "ctx.cuh"

cudaError_t launch_resid_z64(const DevCtx &c, int npts, const z64 *XD, const z64 *X,
                             const z64 *Frow_d, const z64 *Frow_m, const z64 *opg_d,
                             const z64 *opg_m, z32 *V, const z64 *extra_d, unsigned long long *rnorm,
                             const z64 *Bpt, cudaStream_t st);

// X64 = up(Y32) from the RHS columns of the FP32 factorised matrices
__global__ void k_init_x(const z32 *T32, size_t strideM, int N, int R, int nmat, z64 *X) {
  size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  size_t per = (size_t)N * R;
  if (idx >= per * nmat) return;
  size_t m = idx / per, e = idx % per;
  X[idx] = to64(T32[m * strideM + (size_t)N * N + e]);
}

// XD(i1, i3 + nu*nd2) = sum_i2 X(i1, i2 + nu*nd2) sw_nu(i2, i3), row-major R x N
__global__ void k_xd(DevCtx c, int npts, const z64 *X, const z64 *chi0q, const z64 *c0inv, z64 *XD,
                     int minus_one) {
  const int nd2 = c.nd2, N = c.N;
  size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  size_t per = (size_t)nd2 * N;
  if (idx >= per * 2 * npts) return;
  size_t m = idx / per, e = idx % per;
  int i1 = (int)(e / N), col = (int)(e % N);
  int nu = col / nd2, i3 = col % nd2;
  int p = (int)(m >> 1);
  const z64 *x = X + m * per + (size_t)i1 * N + (size_t)nu * nd2;
  const z64 *cq = chi0q + (size_t)p * nd2 * nd2 * 2 * c.iwf + (size_t)nu * nd2 * nd2 + (size_t)i3 * nd2;
  const z64 ci = c0inv[nu * nd2 + i3];
  z64 s = make_double2(0.0, 0.0);
  for (int i2 = 0; i2 < nd2; ++i2) {
    z64 sw = cmul(cq[i2], ci);
    if (i2 == i3 && minus_one) sw.x -= 1.0;
    cfma(s, x[i2], sw);
  }
  XD[m * per + e] = s;
}

// X += up(V); per-matrix max |d| and max |X| (|re|+|im|) into norms[2*m], norms[2*m+1]
__global__ void k_update(int per, const z32 *V, z64 *X, unsigned long long *norms, const int *active) {
  const int m = blockIdx.y;
  if (active && !active[m]) return;
  __shared__ double sd[8], sx[8];
  double md = 0.0, mx = 0.0;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < per; e += gridDim.x * blockDim.x) {
    z64 d = to64(V[(size_t)m * per + e]);
    z64 x = X[(size_t)m * per + e];
    x.x += d.x; x.y += d.y;
    X[(size_t)m * per + e] = x;
    md = fmax(md, fabs(d.x) + fabs(d.y));
    mx = fmax(mx, fabs(x.x) + fabs(x.y));
  }
  for (int o = 16; o > 0; o >>= 1) {
    md = fmax(md, __shfl_xor_sync(0xffffffffu, md, o));
    mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  }
  if ((threadIdx.x & 31) == 0) { sd[threadIdx.x >> 5] = md; sx[threadIdx.x >> 5] = mx; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) { md = fmax(md, sd[w]); mx = fmax(mx, sx[w]); }
    // non-negative doubles order like their bit patterns
    atomicMax(norms + 2 * m, (unsigned long long)__double_as_longlong(md));
    atomicMax(norms + 2 * m + 1, (unsigned long long)__double_as_longlong(mx));
  }
}

cudaError_t launch_init_x(const z32 *T32, size_t strideM, int N, int R, int nmat, z64 *X, cudaStream_t st) {
  size_t total = (size_t)N * R * nmat;
  k_init_x<<<cdiv_u(total, 256), 256, 0, st>>>(T32, strideM, N, R, nmat, X);
  return ADGA_LAUNCH_CHECK();
}

cudaError_t launch_residual(const DevCtx &c, int npts, const z64 *X, const z64 *chi0q,
                            const z64 *c0inv, const z64 *Frow_d, const z64 *Frow_m,
                            const z64 *opg_d, const z64 *opg_m, z64 *XD, z32 *V, const z64 *extra_d,
                            unsigned long long *rnorm, cudaStream_t st, const z64 *Bpt, void *ri8,
                            long long fgen) {
  size_t total = (size_t)c.nd2 * c.N * 2 * npts;
  k_xd<<<cdiv_u(total, 256), 256, 0, st>>>(c, npts, X, chi0q, c0inv, XD, 1);
  cudaError_t e = ADGA_LAUNCH_CHECK();
  if (e != cudaSuccess) return e;
  if (ri8)
    return ri8_residual(ri8, c, npts, XD, X, Frow_d, Frow_m, fgen, opg_d, opg_m, V, extra_d, rnorm, Bpt, st);
  return launch_resid_z64(c, npts, XD, X, Frow_d, Frow_m, opg_d, opg_m, V, extra_d, rnorm, Bpt, st);
}

// XD = X blockdiag(chi0q chi0_loc^-1 - 1), or without the -1 (a tangent direction)
cudaError_t launch_xd(const DevCtx &c, int npts, const z64 *X, const z64 *chi0q, const z64 *c0inv, z64 *XD,
                      bool minus_one, cudaStream_t st) {
  size_t total = (size_t)c.nd2 * c.N * 2 * npts;
  k_xd<<<cdiv_u(total, 256), 256, 0, st>>>(c, npts, X, chi0q, c0inv, XD, minus_one ? 1 : 0);
  return ADGA_LAUNCH_CHECK();
}

cudaError_t launch_update(int per, int nmat, const z32 *V, z64 *X, unsigned long long *norms,
                          const int *active, cudaStream_t st) {
  dim3 g(cdiv_u(per, 256 * 4), nmat);
  k_update<<<g, 256, 0, st>>>(per, V, X, norms, active);
  return ADGA_LAUNCH_CHECK();
}
