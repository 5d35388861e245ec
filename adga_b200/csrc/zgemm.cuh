// Complex FP64 (and FP32) GEMM mainloop on the CUDA cores:
//     acc[8][4] (per thread) = sum_k A(r, k) B(k, c)
// for a 128 x 64 output tile, 256 threads, BK = 8, double-buffered through
// shared memory with cp.async.  Thread (tx, ty) = (t % 16, t / 16) owns rows
// r0 + tx + 16 i (i < 8) and columns c0 + ty + 16 j (j < 4), so that a
// warp's accesses to a column-major C tile are 256-byte contiguous runs.
// Operand access goes through loader functors returning the address of
// A(r, k) / B(k, c) (or nullptr outside the matrix, read as zero).
#pragma once
#include "common.cuh"

namespace zg {

constexpr int BM = 128, BN = 64, BK = 8, TM = 8, TN = 4, NT = 256;

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem, int nbytes) {
  const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(s), "l"(gmem), "r"(nbytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;"); }
__device__ __forceinline__ void cp_async_wait0() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// smem: As[2][BK][BM], Bs[2][BK][BN] of z64 (48 KB).
// A_KFAST: A(r, k) is contiguous in k (row-major A), else in r.
// B_CFAST: B(k, c) is contiguous in c (row-major B), else in k.
// `safe` is any valid global address (source of the zero-filled copies).
template <bool A_KFAST, bool B_CFAST, class LA, class LB>
__device__ __forceinline__ void mainloop(z64 (&acc)[TM][TN], z64 *As, z64 *Bs, int K, const LA &la,
                                         const LB &lb, const z64 *safe) {
  const int t = threadIdx.x, tx = t & 15, ty = t >> 4;
#pragma unroll
  for (int i = 0; i < TM; ++i)
#pragma unroll
    for (int j = 0; j < TN; ++j) acc[i][j] = make_double2(0.0, 0.0);
  auto load = [&](int stage, int k0) {
    z64 *as = As + stage * BK * BM, *bs = Bs + stage * BK * BN;
#pragma unroll
    for (int q = 0; q < (BM * BK) / NT; ++q) {          // 4 per thread
      const int e = t + NT * q;
      const int r = A_KFAST ? e / BK : e % BM, kk = A_KFAST ? e % BK : e / BM;
      const z64 *g = la(r, k0 + kk);
      cp_async16(as + kk * BM + r, g ? g : safe, g ? 16 : 0);
    }
#pragma unroll
    for (int q = 0; q < (BN * BK) / NT; ++q) {          // 2 per thread
      const int e = t + NT * q;
      const int kk = B_CFAST ? e / BN : e % BK, c = B_CFAST ? e % BN : e / BK;
      const z64 *g = lb(k0 + kk, c);
      cp_async16(bs + kk * BN + c, g ? g : safe, g ? 16 : 0);
    }
    cp_async_commit();
  };
  const int nk = (K + BK - 1) / BK;
  if (nk == 0) return;
  load(0, 0);
  for (int kt = 0; kt < nk; ++kt) {
    cp_async_wait0();
    __syncthreads();
    if (kt + 1 < nk) load((kt + 1) & 1, (kt + 1) * BK);
    const z64 *as = As + (kt & 1) * BK * BM, *bs = Bs + (kt & 1) * BK * BN;
#pragma unroll
    for (int kk = 0; kk < BK; ++kk) {
      z64 a[TM], b[TN];
#pragma unroll
      for (int i = 0; i < TM; ++i) a[i] = as[kk * BM + tx + 16 * i];
#pragma unroll
      for (int j = 0; j < TN; ++j) b[j] = bs[kk * BN + ty + 16 * j];
#pragma unroll
      for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int j = 0; j < TN; ++j) cfma(acc[i][j], a[i], b[j]);
    }
    __syncthreads();
  }
}

}  // namespace zg
