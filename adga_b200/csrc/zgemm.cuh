// Complex FP64 GEMM mainloop on the CUDA cores:
//     acc[8][4] (per thread) = sum_k A(r, k) B(k, c)
// for a 128 x 64 output tile, 256 threads, k-slices of BK = 16 through a
// STAGES-deep cp.async ring in shared memory (one barrier per slice).
// Thread (tx, ty) = (t % 16, t / 16) owns rows r0 + tx + 16 i (i < 8) and
// columns c0 + ty + 16 j (j < 4), so that a warp's accesses to a
// column-major C tile are 256-byte contiguous runs.  Operand access goes
// through loader functors returning the address of A(r, k) / B(k, c) (or
// nullptr outside the matrix, read as zero).
#pragma once
#include "common.cuh"

namespace zg {

constexpr int BM = 128, BN = 64, BK = 16, TM = 8, TN = 4, NT = 256, STAGES = 3;
// dynamic shared memory of a kernel built on mainloop: As[STAGES][BK][BM], Bs[STAGES][BK][BN]
constexpr int SMEM_BYTES = STAGES * BK * (BM + BN) * 16;

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem, int nbytes) {
  const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(s), "l"(gmem), "r"(nbytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;"); }
template <int N> __device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

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
  const int nk = (K + BK - 1) / BK;
  auto load = [&](int kt) {
    if (kt < nk) {
      const int stage = kt % STAGES, k0 = kt * BK;
      z64 *as = As + stage * BK * BM, *bs = Bs + stage * BK * BN;
#pragma unroll
      for (int q = 0; q < (BM * BK) / NT; ++q) {          // 8 per thread
        const int e = t + NT * q;
        const int r = A_KFAST ? e / BK : e % BM, kk = A_KFAST ? e % BK : e / BM;
        const z64 *g = la(r, k0 + kk);
        cp_async16(as + kk * BM + r, g ? g : safe, g ? 16 : 0);
      }
#pragma unroll
      for (int q = 0; q < (BN * BK) / NT; ++q) {          // 4 per thread
        const int e = t + NT * q;
        const int kk = B_CFAST ? e / BN : e % BK, c = B_CFAST ? e % BN : e / BK;
        const z64 *g = lb(k0 + kk, c);
        cp_async16(bs + kk * BN + c, g ? g : safe, g ? 16 : 0);
      }
    }
    cp_async_commit();
  };
  if (nk == 0) return;
#pragma unroll
  for (int s = 0; s < STAGES - 1; ++s) load(s);
  for (int kt = 0; kt < nk; ++kt) {
    cp_async_wait<STAGES - 2>();
    __syncthreads();                 // slice kt landed; slice kt-1's stage is free
    load(kt + STAGES - 1);
    const z64 *as = As + (kt % STAGES) * BK * BM, *bs = Bs + (kt % STAGES) * BK * BN;
#pragma unroll 4
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
  }
  cp_async_wait<0>();
}

}  // namespace zg
