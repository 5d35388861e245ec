// Tensor-core (tcgen05) trailing update of the mixed-precision BSE LU:
//     C -= L21 * U12        (complex FP32 storage, per matrix of the batch)
// computed as a real BF16 GEMM with FP32 accumulation in TMEM using the
// 3-term split x = x_hi + x_lo (x_hi = bf16(x), x_lo = bf16(x - x_hi)):
//     L U ~= L_hi U_hi + L_hi U_lo + L_lo U_hi .
// Complex arithmetic is embedded as
//     [Re C | Im C] = [Lr | Li] . [[Ur, Ui], [-Ui, Ur]]
// so two MMAs of N = BN produce the real (columns 0..BN) and imaginary
// (BN..2BN) parts of BN complex columns.  Operands are staged per step in
// K-major BF16, four segments of NB each (K4 = 4*NB per step):
//     A[m]     = [Lr_hi, Li_hi, Lr_lo, Li_lo]
//     Bre[n]   = [Ur_hi, -Ui_hi, Ur_lo, -Ui_lo]
// and the GEMMs run six segment pairs per step (A, B) = (0,0), (1,1), (0,2),
// (1,3), (2,0), (3,1): the hi*hi, hi*lo and lo*hi products of the real and
// imaginary parts (K = 6*NB of MMAs from 4*NB of staging).  The rows of
// [Ui, Ur], Bim[n] = [Ui_hi, Ur_hi, Ui_lo, Ur_lo], are segment s ^ 1 of
// Bre[n], negated for even s: the imaginary-part MMA reads them from the
// real-part staging with the instruction's B negation, so only Bre is staged.
// (TMA loads, 128B swizzle, into a ring of shared-memory stages; tcgen05.mma
// M=128, N=128, K=16 issued by one thread, FP32 accumulators in TMEM):
//   k_tc_persist  (used when the C strides are 16-byte multiples) one CTA per
//                 SM loops over the tiles; C tiles arrive in shared memory by
//                 TMA during the MMAs and the accumulator is double-buffered,
//                 so the C read-modify-write overlaps the next tile;
//   k_tc_update   one CTA per tile, C read and written by the epilogue warps.
// Every mbarrier wait is bounded; on timeout the kernel records an error and
// leaves.  Loads use no cluster multicast.
#include "lu.cuh"
#include "umma.cuh"
#include <cuda.h>
#include <cuda_bf16.h>
#include <algorithm>
#include <cstdio>

namespace {

using namespace umma;

constexpr int BM = 128;          // rows per tile (MMA M)
constexpr int BN = 128;          // complex columns per tile (MMA N = 2*BN)
constexpr int BK = 64;           // bf16 per stage row (one 128 B swizzle atom)
constexpr int STAGES = 2;
constexpr int A_BYTES = BM * BK * 2;           // 16 KB
constexpr int B_BYTES = 2 * BN * BK * 2;       // 32 KB
constexpr int STAGE_BYTES = A_BYTES + B_BYTES;
constexpr int TMEM_COLS = 2 * BN;              // 256 fp32 columns
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024 + 256;
// the staging segments of MMA k-segment j (0..5) of a step: A and B segment indices
__device__ __forceinline__ int seg_a(int j) { return j < 4 ? (j & 1) : j - 2; }
__device__ __forceinline__ int seg_b(int j) { return j < 4 ? j : j - 4; }
// x coordinate (bf16) in the four-segment staging of k-block kb of a step (nbk = NB / BK)
__device__ __forceinline__ int kx_a(int kb, int nbk) { return (seg_a(kb / nbk) * nbk + kb % nbk) * BK; }
__device__ __forceinline__ int kx_b(int kb, int nbk) { return (seg_b(kb / nbk) * nbk + kb % nbk) * BK; }
// B's imaginary-part rows [Ui_hi, Ur_hi, Ui_lo, Ur_lo] are not staged: segment s of such a row is
// segment s ^ 1 of the real-part row [Ur_hi, -Ui_hi, Ur_lo, -Ui_lo], negated for even s; the
// k-block's x coordinate in the real-part staging, and whether its MMA negates B
__device__ __forceinline__ int kx_bi(int kb, int nbk) { return ((seg_b(kb / nbk) ^ 1) * nbk + kb % nbk) * BK; }
__device__ __forceinline__ uint32_t neg_bi(int kb, int nbk) { return (seg_b(kb / nbk) & 1) ? 0u : 1u; }
// K-major, 128 B swizzle: LBO = 16 B (unused), SBO = 1024 B between 8-row groups
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
  uint64_t d = 0;
  d |= (uint64_t)((addr & 0x3FFFF) >> 4);
  d |= (uint64_t)1 << 16;                 // leading byte offset (16 B units)
  d |= (uint64_t)(1024 >> 4) << 32;       // stride byte offset
  d |= (uint64_t)1 << 46;                 // descriptor version (sm_100)
  d |= (uint64_t)2 << 61;                 // SWIZZLE_128B
  return d;
}
// kind::f16, A = B = BF16, D = F32, both K-major, M = 128, N = 128 (bit 14: negate B)
constexpr uint32_t IDESC_H = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN / 8) << 17) |
                             ((uint32_t)(BM / 16) << 24);

__device__ __forceinline__ void mma_bf16_h(uint32_t tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(acc));
}
// one K = 16 slice of a k-block into [Re C | Im C]: the real-part columns from B's first 128
// rows, the imaginary-part columns from the second 128 (B negated when neg)
__device__ __forceinline__ void mma_cplx(uint32_t tmem, uint32_t sa, uint32_t sb, uint32_t neg, uint32_t acc,
                                         uint32_t idesc = IDESC_H) {
  mma_bf16_h(tmem, smem_desc(sa), smem_desc(sb), idesc, acc);
  mma_bf16_h(tmem + BN, smem_desc(sa), smem_desc(sb + B_BYTES / 2), idesc | (neg << 14), acc);
}
// the same with N = 64: a tile with at most 64 columns inside the region (the narrow strips)
constexpr uint32_t IDESC_Q = (IDESC_H & ~(0x3Fu << 17)) | ((uint32_t)(64 / 8) << 17);
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(192, 2)
k_tc_update(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB,
            z32 *M, size_t strideM, int N, int J, int jb, int Mrows, int Ncols, int Ncap, int nkb,
            int b0, int nbk, int *err) {
  extern __shared__ unsigned char smraw[];
  const uint32_t sbase = (smem_u32(smraw) + 1023u) & ~1023u;
  unsigned char *gbase = smraw + (sbase - smem_u32(smraw));
  uint64_t *bars = reinterpret_cast<uint64_t *>(gbase + STAGES * STAGE_BYTES);
  uint32_t *tslot = reinterpret_cast<uint32_t *>(bars + 2 * STAGES + 1);
  const uint32_t bar_full = smem_u32(bars), bar_empty = bar_full + 8 * STAGES,
                 bar_acc = bar_full + 16 * STAGES;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int n0 = blockIdx.x * BN, m0 = blockIdx.y * BM, b = b0 + blockIdx.z;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(bar_full + 8 * s, 1);
      mbar_init(bar_empty + 8 * s, 1);
    }
    mbar_init(bar_acc, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                 "r"(TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = *tslot;
  bool ok = true;

  if (warp == 0) {
    if (lane == 0) {
      for (int kb = 0; kb < nkb && ok; ++kb) {
        const int s = kb % STAGES;
        if (kb >= STAGES) ok = mbar_wait(bar_empty + 8 * s, ((kb / STAGES) - 1) & 1, err, 1);
        if (!ok) break;
        const uint32_t sa = sbase + s * STAGE_BYTES, sb = sa + A_BYTES;
        mbar_expect_tx(bar_full + 8 * s, STAGE_BYTES);
        tma_load_3d(sa, &mapA, bar_full + 8 * s, kx_a(kb, nbk), m0, b);
        tma_load_3d(sb, &mapB, bar_full + 8 * s, kx_b(kb, nbk), n0, b);
        tma_load_3d(sb + B_BYTES / 2, &mapB, bar_full + 8 * s, kx_bi(kb, nbk), n0, b);
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      for (int kb = 0; kb < nkb && ok; ++kb) {
        const int s = kb % STAGES;
        ok = mbar_wait(bar_full + 8 * s, (kb / STAGES) & 1, err, 2);
        if (!ok) break;
        asm volatile("tcgen05.fence::after_thread_sync;");
        const uint32_t sa = sbase + s * STAGE_BYTES, sb = sa + A_BYTES;
        const uint32_t neg = neg_bi(kb, nbk);
#pragma unroll
        for (int k = 0; k < BK / 16; ++k) mma_cplx(tmem, sa + 32 * k, sb + 32 * k, neg, (kb > 0 || k > 0) ? 1u : 0u);
        mma_commit(bar_empty + 8 * s);
      }
      mma_commit(bar_acc);
    }
  } else {
    // epilogue: warp w reads TMEM lanes 32*(w%4).. (= tile rows)
    const int quad = warp & 3;
    const int row = quad * 32 + lane;
    ok = __all_sync(0xffffffffu, mbar_wait(bar_acc, 0, err, 3));
    asm volatile("tcgen05.fence::after_thread_sync;");
    if (ok) {
      const int m = m0 + row;
      z32 *Cb = M + (size_t)b * strideM + (size_t)(J + jb + m);
      const uint32_t tl = tmem + ((uint32_t)(quad * 32) << 16);
      const bool rowok = m < Mrows;
      // Each C element is read once and then written by this thread only, so
      // the loads go through the read-only path and are issued a chunk ahead
      // of the stores (software pipelining over 16-column chunks).
      auto ldc = [&](int c, z32 (&cv)[16]) {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int n = n0 + c + j;
          cv[j] = (rowok && n < Ncols) ? __ldg(Cb + (size_t)(J + jb + n) * N) : make_float2(0.f, 0.f);
        }
      };
      z32 cur[16], nxt[16];
      ldc(0, cur);
#pragma unroll 1
      for (int c = 0; c < BN; c += 16) {
        if (c + 16 < BN) ldc(c + 16, nxt);
        float re[16], im[16];
        tmem_ld16(tl + c, re);
        tmem_ld16(tl + BN + c, im);
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int n = n0 + c + j;
          if (rowok && n < Ncols) {
            z32 v = cur[j];
            v.x -= re[j];
            v.y -= im[j];
            Cb[(size_t)(J + jb + n) * N] = v;
          }
        }
#pragma unroll
        for (int j = 0; j < 16; ++j) cur[j] = nxt[j];
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 1) {
    // every MMA has completed once bar_acc fired; on an error path the MMA
    // thread issued no further work after its last commit
    asm volatile("tcgen05.fence::after_thread_sync;");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS));
  }
}

// ---------------------------------------------------------------------------
// Persistent variant: one CTA per SM loops over the (column tile, row tile,
// matrix) tiles of the launch; the accumulator is double-buffered in TMEM
// (2 x 256 columns), so the epilogue of one tile overlaps the loads and MMAs
// of the next.  Operands: the six k-segment products of a step's K = 64 use
// only four A and four B segments (A = [Lr_hi, Li_hi, Lr_lo, Li_lo], B =
// [Ur_hi, -Ui_hi, Ur_lo, -Ui_lo]; product j multiplies A segment seg_a(j)
// by B segments seg_b(j) (real part) and seg_b(j) ^ 1 (imaginary part)), so
// each 16 KB operand tile is loaded once per step and tile and serves two or
// four products.  The tiles travel in pairs through a ring of five 32 KB
// slots, in the order [B2 B3] [A0 A1] [B0 B1] [A2 A3]; the products run in
// the order j = 2, 3 (first two slots), 0, 1 (third), 4, 5 (fourth), which
// frees the slots in the order they were filled.  128 KB of operands per
// tile and step feed 48 MMAs (M = 128, N = 128, K = 16).  The C tile reaches
// shared memory by TMA one 64-column half at a time through one 64 KB buffer
// (the second half is prefetched into L2 when the first is loaded).
//   warp 0        TMA loads of the operand pairs (ring of P_SLOTS)
//   warp 1        TMEM allocation (512 columns) and tcgen05.mma issue
//   warp 2        TMA loads of the C halves
//   warps 4..11   epilogue: per half, group g = 0, 1 owns its columns 32 g..,
//                 warp w reads TMEM lanes 32*(w%4)..; C - acc is stored
//                 straight to global
// Every wait is bounded (WAIT_NS); on a timeout a role records an error and
// stops issuing work.
// ---------------------------------------------------------------------------
constexpr int P_SLOTS = 5;                            // operand ring: slots of two tiles
constexpr int P_TILE = BM * BK * 2;                   // one 128-row x 64-bf16 operand tile: 16 KB
constexpr int P_PAIR = 2 * P_TILE;                    // a slot: two segments of A or of B
constexpr int P_CH_COLS = 64;                         // columns per C half
constexpr int P_CH_BYTES = BM * 8 * P_CH_COLS;        // 64 KB of complex FP32
constexpr int P_TMEM_COLS = 2 * TMEM_COLS;            // two accumulators
constexpr int P_THREADS = 384;
constexpr int P_SMEM_BYTES = P_SLOTS * P_PAIR + P_CH_BYTES + 1024 + 256;
static_assert(BN == BM, "A and B operand tiles share one box");
static_assert(P_SMEM_BYTES <= 232448, "shared memory of one CTA");

__device__ __forceinline__ void tma_prefetch_l2_3d(const CUtensorMap *map, int x, int y, int z) {
  asm volatile("cp.async.bulk.prefetch.tensor.3d.L2.global.tile [%0, {%1, %2, %3}];" ::"l"(
                   (unsigned long long)map),
               "r"(x), "r"(y), "r"(z)
               : "memory");
}

// the four K = 16 slices of one product: A tile sa into [Re C | Im C], the real-part
// columns from B tile sre, the imaginary-part columns from B tile sim (negated when neg)
__device__ __forceinline__ void mma_prod(uint32_t dacc, uint32_t sa, uint32_t sre, uint32_t sim, uint32_t neg,
                                         bool first, uint32_t idesc) {
#pragma unroll
  for (int k = 0; k < BK / 16; ++k) {
    const uint32_t acc = (first && k == 0) ? 0u : 1u;
    mma_bf16_h(dacc, smem_desc(sa + 32 * k), smem_desc(sre + 32 * k), idesc, acc);
    mma_bf16_h(dacc + BN, smem_desc(sa + 32 * k), smem_desc(sim + 32 * k), idesc | (neg << 14), acc);
  }
}

// the tensor maps of up to four operand stagings (the steps of a delayed group) and of C,
// and each staging's row / column offset for the region's first C row / column
constexpr int P_MAXST = 4;
struct alignas(64) PMaps {
  CUtensorMap a[P_MAXST], b[P_MAXST], c, c64;   // c64: C halves of 64 rows (regions of at most 64 rows)
};
struct POff {
  int ar[P_MAXST], bc[P_MAXST];
};

__global__ void __launch_bounds__(P_THREADS, 1)
k_tc_persist(const __grid_constant__ PMaps maps, z32 *M, size_t strideM, int N, int crow0, int ccol0, POff off,
             int nst, int nbk, int Mrows, int Ncols, int b0, int count, int *err) {
  extern __shared__ unsigned char smraw[];
  const uint32_t sbase = (smem_u32(smraw) + 1023u) & ~1023u;
  unsigned char *gbase = smraw + (sbase - smem_u32(smraw));
  const uint32_t scbase = sbase + P_SLOTS * P_PAIR;                 // the C half buffer
  const unsigned char *gc = gbase + P_SLOTS * P_PAIR;
  uint64_t *bars = reinterpret_cast<uint64_t *>(gbase + P_SLOTS * P_PAIR + P_CH_BYTES);
  uint32_t *tslot = reinterpret_cast<uint32_t *>(bars + 2 * P_SLOTS + 8);
  const uint32_t bar_full = smem_u32(bars), bar_empty = bar_full + 8 * P_SLOTS;
  const uint32_t bar_accf = bar_empty + 8 * P_SLOTS;    // [2]
  const uint32_t bar_acce = bar_accf + 16;              // [2]
  const uint32_t bar_cfull = bar_acce + 16;             // [2]
  const uint32_t bar_cempty = bar_cfull + 16;           // [2]
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ntn = (Ncols + BN - 1) / BN, ntm = (Mrows + BM - 1) / BM;
  const int ntiles = ntn * ntm * count;
  const int nunit = nst * nbk;                          // (staging, k-block) units per tile

  if (threadIdx.x == 0) {
    for (int s = 0; s < P_SLOTS; ++s) {
      mbar_init(bar_full + 8 * s, 1);
      mbar_init(bar_empty + 8 * s, 1);
    }
    for (int a = 0; a < 2; ++a) {
      mbar_init(bar_accf + 8 * a, 1);
      mbar_init(bar_acce + 8 * a, 8);      // one arrival per epilogue warp
    }
    mbar_init(bar_cfull, 1);
    mbar_init(bar_cempty, 8);              // one arrival per epilogue warp
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                 "r"(P_TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = *tslot;

  if (warp == 0) {
    if (lane == 0) {
      int pt = 0;     // slot fills so far
      bool ok = true;
      for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
        const int tn = tile % ntn, tm = (tile / ntn) % ntm, b = b0 + tile / (ntn * ntm);
        for (int u = 0; u < nunit && ok; ++u) {
          const int sti = u / nbk, kk = u - sti * nbk;
          const CUtensorMap *ma = &maps.a[sti], *mb = &maps.b[sti];
          const int ya = (sti == 0 ? off.ar[0] : sti == 1 ? off.ar[1] : sti == 2 ? off.ar[2] : off.ar[3]) + tm * BM;
          const int yb = (sti == 0 ? off.bc[0] : sti == 1 ? off.bc[1] : sti == 2 ? off.bc[2] : off.bc[3]) + tn * BN;
          // slot q: [B2 B3], [A0 A1], [B0 B1], [A2 A3]; segment s of k-block kk at x = (s nbk + kk) BK
#pragma unroll 1
          for (int q = 0; q < 4; ++q, ++pt) {
            const int s = pt % P_SLOTS;
            if (pt >= P_SLOTS && !(ok = mbar_wait(bar_empty + 8 * s, ((pt / P_SLOTS) - 1) & 1, err, 11))) break;
            const uint32_t d = sbase + s * P_PAIR;
            const bool isa = q & 1;
            const int seg = (q == 0 || q == 3) ? 2 : 0;
            const CUtensorMap *m = isa ? ma : mb;
            const int y = isa ? ya : yb;
            mbar_expect_tx(bar_full + 8 * s, P_PAIR);
            tma_load_3d(d, m, bar_full + 8 * s, (seg * nbk + kk) * BK, y, b);
            tma_load_3d(d + P_TILE, m, bar_full + 8 * s, ((seg + 1) * nbk + kk) * BK, y, b);
          }
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      int pt = 0, it = 0;
      bool ok = true;
      for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x, ++it) {
        const int a = it & 1, use = it >> 1;
        if (use > 0 && !(ok = mbar_wait(bar_acce + 8 * a, (use - 1) & 1, err, 12))) break;
        asm volatile("tcgen05.fence::after_thread_sync;");
        const uint32_t dacc = tmem + (uint32_t)(a * TMEM_COLS);
        const uint32_t idesc = Ncols - (tile % ntn) * BN <= 64 ? IDESC_Q : IDESC_H;
        for (int u = 0; u < nunit; ++u, pt += 4) {
          const int s0 = pt % P_SLOTS, s1 = (pt + 1) % P_SLOTS, s2 = (pt + 2) % P_SLOTS, s3 = (pt + 3) % P_SLOTS;
          const uint32_t b23 = sbase + s0 * P_PAIR, a01 = sbase + s1 * P_PAIR;
          const uint32_t b01 = sbase + s2 * P_PAIR, a23 = sbase + s3 * P_PAIR;
          if (!(ok = mbar_wait(bar_full + 8 * s0, (pt / P_SLOTS) & 1, err, 13) &&
                     mbar_wait(bar_full + 8 * s1, ((pt + 1) / P_SLOTS) & 1, err, 13)))
            break;
          asm volatile("tcgen05.fence::after_thread_sync;");
          mma_prod(dacc, a01, b23, b23 + P_TILE, 1u, u == 0, idesc);            // j = 2: A0 x (B2, -B3)
          mma_prod(dacc, a01 + P_TILE, b23 + P_TILE, b23, 0u, false, idesc);    // j = 3: A1 x (B3, B2)
          mma_commit(bar_empty + 8 * s0);
          if (!(ok = mbar_wait(bar_full + 8 * s2, ((pt + 2) / P_SLOTS) & 1, err, 13))) break;
          asm volatile("tcgen05.fence::after_thread_sync;");
          mma_prod(dacc, a01, b01, b01 + P_TILE, 1u, false, idesc);             // j = 0: A0 x (B0, -B1)
          mma_prod(dacc, a01 + P_TILE, b01 + P_TILE, b01, 0u, false, idesc);    // j = 1: A1 x (B1, B0)
          mma_commit(bar_empty + 8 * s1);
          if (!(ok = mbar_wait(bar_full + 8 * s3, ((pt + 3) / P_SLOTS) & 1, err, 13))) break;
          asm volatile("tcgen05.fence::after_thread_sync;");
          mma_prod(dacc, a23, b01, b01 + P_TILE, 1u, false, idesc);             // j = 4: A2 x (B0, -B1)
          mma_prod(dacc, a23 + P_TILE, b01 + P_TILE, b01, 0u, false, idesc);    // j = 5: A3 x (B1, B0)
          mma_commit(bar_empty + 8 * s2);
          mma_commit(bar_empty + 8 * s3);
        }
        if (!ok) break;
        mma_commit(bar_accf + 8 * a);
      }
    }
  } else if (warp == 2) {
    if (lane == 0) {
      int it = 0;
      int u = 0;     // uses of the one C buffer so far (halves with columns inside the region)
      for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++it) {
        const int tn = tile % ntn, tm = (tile / ntn) % ntm, b = b0 + tile / (ntn * ntm);
        bool ok = true;
        for (int h = 0; h < 2 && ok; ++h) {
          if (tn * BN + h * P_CH_COLS >= Ncols) break;   // the half lies outside the region
          // the epilogue has released use u - 1
          if (u > 0) ok = mbar_wait(bar_cempty, (u - 1) & 1, err, 14);
          if (!ok) break;
          ++u;
          // a region of at most 64 rows (the next step's rows in a delayed group) loads only those
          const bool r64 = Mrows <= 64;
          const CUtensorMap *mc = r64 ? &maps.c64 : &maps.c;
          mbar_expect_tx(bar_cfull, r64 ? P_CH_BYTES / 2 : P_CH_BYTES);
          // x counts floats: rows crow0 + m.. as (re, im) pairs (crow0 even: 16-byte aligned)
          tma_load_3d(scbase, mc, bar_cfull, 2 * (crow0 + tm * BM), ccol0 + tn * BN + h * P_CH_COLS, b);
          if (h == 0 && tn * BN + P_CH_COLS < Ncols)
            tma_prefetch_l2_3d(mc, 2 * (crow0 + tm * BM), ccol0 + tn * BN + P_CH_COLS, b);
        }
        if (!ok) break;
      }
    }
  } else if (warp >= 4) {
    const int e = warp - 4, grp = e >> 2, quad = warp & 3;
    const int row = quad * 32 + lane;
    const z32 *cs = reinterpret_cast<const z32 *>(gc);   // [col][128 rows] of the current half
    int it = 0, u = 0;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++it) {
      const int tn = tile % ntn, tm = (tile / ntn) % ntm, b = b0 + tile / (ntn * ntm);
      const int a = it & 1;
      // the warp leaves together if any lane gave up, so tcgen05.ld stays warp-wide
      bool ok = mbar_wait(bar_accf + 8 * a, (it >> 1) & 1, err, 15);
      if (!__all_sync(0xffffffffu, ok)) break;
      asm volatile("tcgen05.fence::after_thread_sync;");
      const int m = tm * BM + row;
      const bool rowok = m < Mrows;
      const int cld = Mrows <= 64 ? 64 : BM;     // rows per column of the C half in shared memory
      z32 *Cb = M + (size_t)b * strideM + (size_t)(crow0 + m);
      for (int h = 0; h < 2 && ok; ++h) {
        if (tn * BN + h * P_CH_COLS >= Ncols) break;     // no C loaded: outside the region
        // every lane waits (and so observes the TMA-written C half)
        ok = mbar_wait(bar_cfull, u & 1, err, 16);
        ++u;
        if (!__all_sync(0xffffffffu, ok)) { ok = false; break; }
        const int c0 = h * P_CH_COLS + grp * 32;            // accumulator column of this warp's part
        const uint32_t tl = tmem + ((uint32_t)(quad * 32) << 16) + (uint32_t)(a * TMEM_COLS + c0);
        const int nbase = tn * BN + c0;
#pragma unroll 1
        for (int c = 0; c < 32; c += 16) {
          float re[16], im[16];
          tmem_ld16(tl + c, re);
          tmem_ld16(tl + BN + c, im);
          z32 cv[16];
#pragma unroll
          for (int j = 0; j < 16; ++j) cv[j] = cs[(grp * 32 + c + j) * cld + (rowok ? row : 0)];
          asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
          for (int j = 0; j < 16; ++j) {
            const int n = nbase + c + j;
            if (rowok && n < Ncols) {
              z32 v = cv[j];
              v.x -= re[j];
              v.y -= im[j];
              Cb[(size_t)(ccol0 + n) * N] = v;
            }
          }
        }
        // this warp is done with the C half
        __syncwarp();
        if (lane == 0) mbar_arrive(bar_cempty);
      }
      if (!ok) break;
      // and with the accumulator
      asm volatile("tcgen05.fence::before_thread_sync;");
      __syncwarp();
      if (lane == 0) mbar_arrive(bar_acce + 8 * a);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 1) {
    asm volatile("tcgen05.fence::after_thread_sync;");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(P_TMEM_COLS));
  }
}

// ---------------------------------------------------------------------------
// operand staging
// ---------------------------------------------------------------------------
__device__ __forceinline__ void split2(float x, __nv_bfloat16 &hi, __nv_bfloat16 &lo) {
  hi = __float2bfloat16_rn(x);
  lo = __float2bfloat16_rn(x - __bfloat162float(hi));
}

// ---------------------------------------------------------------------------
// Panel products of one unpivoted step on the tensor cores (k_tc_tri):
//   mode 0   L21   = A21 U11^-1     rows J+jb.. of the step's jb columns
//   mode 1   U12^T = A12^T L11^-T   columns J+jb.. (right-hand sides included)
//                                   of the step's jb rows
// with U11^-1 / L11^-1 the 64 x 64 block inverses of k_diag_inv.  One CTA per
// tile of 128 rows (mode 0) or 128 columns (mode 1) of one matrix, K = 64:
//   * every thread (512 per CTA, two CTAs per SM) loads its 16 values of the
//     FP32 tile from the matrix (coalesced), splits each into bf16 hi + lo
//     and writes the K-major, 128 B swizzled A operand;
//   * the block inverse W becomes the B operand once, rows [Wr(:, n)] and
//     [Wi(:, n)], hi and lo K blocks (mode 0 stages W through shared memory
//     so that its column-major reads are coalesced);
//   * one thread issues the (hi, hi), (hi, lo) and (lo, hi) products of the
//     3-term split into one TMEM accumulator (columns 0..63 real, 64..127
//     imaginary parts): the real part of the tile times [Wr | Wi] (M = 128,
//     N = 128, K = 16), then its imaginary part times [-Wi | Wr] as two N = 64
//     MMAs over B's swapped halves (B negation for the real part);
//   * the epilogue (thread = row of the tile) writes the FP32 result into the
//     matrix and the step's operand staging of the trailing update
//     (k_split_a's layout for L21, k_split_b's for U12), so no split kernel
//     runs for the step: L21's FP32 rows straight from registers, the staging
//     rows and U12's FP32 columns through 128 B swizzled boxes in the freed
//     operand region, stored by TMA;
//   * each thread first prefetches one line of the tile into L2, so that the
//     tile's DRAM latency overlaps the B build.
// The wait on the MMAs is bounded (WAIT_NS); on a timeout the CTA records an
// error and skips its epilogue.
// ---------------------------------------------------------------------------
constexpr int TT_THREADS = 512;
constexpr int TT_ROWS = 128;                       // tile rows (MMA M)
constexpr int TT_KBLK = TT_ROWS * 128;             // one K block: 128 rows x 64 bf16
constexpr int TT_OPER = 4 * TT_KBLK;               // A hi, A lo, B hi, B lo of one K half: 64 KB
constexpr int TT_BOX = TT_ROWS * 128;              // one 128 B swizzled store box: 128 rows x 128 B
constexpr int TT_REGION = TT_OPER;                 // operands, then the epilogue's four store boxes
constexpr int TT_SMEM_BYTES = TT_REGION + 1024 + 64;
static_assert(4 * TT_BOX == TT_OPER, "the epilogue's boxes reuse the operand region");
constexpr int TT_TMEM_COLS = 128;
// kind::f16, A = B = BF16, D = F32, both K-major, M = 128, N = 128
constexpr uint32_t IDESC_N128 = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(128 / 8) << 17) |
                                ((uint32_t)(TT_ROWS / 16) << 24);

// the same with N = 64 (bit 14: negate B)
constexpr uint32_t IDESC_N64 = (IDESC_N128 & ~(0x3Fu << 17)) | ((uint32_t)(64 / 8) << 17);

__device__ __forceinline__ void mma_bf16_tt(uint32_t tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(acc));
}
// byte offset of 16-byte chunk c (0..7) of row r in a 128 B swizzled K block
__device__ __forceinline__ uint32_t sw128(int r, int c) {
  return (uint32_t)((r >> 3) * 1024 + (r & 7) * 128 + ((c ^ (r & 7)) << 4));
}
__device__ __forceinline__ uint32_t pack_bf16(__nv_bfloat16 a, __nv_bfloat16 b) {
  return (uint32_t)__bfloat16_as_ushort(a) | ((uint32_t)__bfloat16_as_ushort(b) << 16);
}
// 8 consecutive K values of one row -> chunk c of the hi block (at base) and of the lo block
// (at base + TT_KBLK), scaled by sgn
__device__ __forceinline__ void put8(unsigned char *base, int r, int c, const float *x, float sgn) {
  uint32_t hw[4], lw[4];
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    __nv_bfloat16 h0, l0, h1, l1;
    split2(sgn * x[2 * u], h0, l0);
    split2(sgn * x[2 * u + 1], h1, l1);
    hw[u] = pack_bf16(h0, h1);
    lw[u] = pack_bf16(l0, l1);
  }
  const uint32_t off = sw128(r, c);
  *reinterpret_cast<uint4 *>(base + off) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
  *reinterpret_cast<uint4 *>(base + TT_KBLK + off) = make_uint4(lw[0], lw[1], lw[2], lw[3]);
}
// 8 bf16 of the values x[0..7] (split part `part`: 0 re hi, 1 re lo, 2 im hi, 3 im lo), negated when neg
__device__ __forceinline__ uint4 pack8(const float *re, const float *im, int part, bool neg) {
  uint32_t w[4];
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    __nv_bfloat16 p2[2];
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      __nv_bfloat16 hi, lo;
      split2(part < 2 ? re[2 * u + e] : im[2 * u + e], hi, lo);
      p2[e] = (part & 1) ? lo : hi;
      if (neg) p2[e] = __hneg(p2[e]);
    }
    w[u] = pack_bf16(p2[0], p2[1]);
  }
  return make_uint4(w[0], w[1], w[2], w[3]);
}

// the step's operand stagings (L21 rows: A, U12 columns: B) and U12 as FP32 columns, all with
// 128 B swizzled boxes of 128 rows x 128 B: the epilogue's TMA stores
struct alignas(64) TriMaps {
  CUtensorMap stA, stB, u;
};

// Panel products (see the block comment above).  The complex product
// [Cr | Ci] = Xr [Wr | Wi] + Xi [-Wi | Wr] runs as two MMA phases over the
// real and the imaginary part of X with one B operand (64 KB of operands at
// a time, so two CTAs share an SM and the load, MMA and store phases of
// different tiles overlap); the epilogue stages all 128 tile rows per round
// in the same shared memory (67.6 KB).
__global__ void __launch_bounds__(TT_THREADS, 2)
k_tc_tri(const __grid_constant__ TriMaps maps, z32 *M, size_t strideM, int N, int ncols, int J, int jb, int NB,
         int nsteps, const z32 *Linv, const z32 *Uinv, int b0, int ntA, int ntU, int *err) {
  extern __shared__ unsigned char smraw[];
  const uint32_t sbase = (smem_u32(smraw) + 1023u) & ~1023u;
  unsigned char *gA = smraw + (sbase - smem_u32(smraw));    // A hi, A lo, B hi, B lo
  unsigned char *gB = gA + 2 * TT_KBLK;
  uint64_t *bar = reinterpret_cast<uint64_t *>(gA + TT_REGION);
  uint32_t *tslot = reinterpret_cast<uint32_t *>(bar + 1);
  const uint32_t sA = sbase, sB = sbase + 2 * TT_KBLK, sbar = smem_u32(bar);
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const int per = ntA + ntU;
  const int b = b0 + blockIdx.x / per, tile = blockIdx.x % per;
  const bool lower = tile < ntA;                       // mode 0: L21
  const int m0 = (lower ? tile : tile - ntA) * TT_ROWS;
  const int nrows = lower ? N - J - jb : ncols - J - jb;
  const int nv = min(TT_ROWS, nrows - m0);             // valid rows of the tile
  z32 *Am = M + (size_t)b * strideM;
  const z32 *W = (lower ? Uinv : Linv) + ((size_t)b * nsteps + J / NB) * NB * NB;

  if (t == 0) {
    mbar_init(sbar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                 "r"(TT_TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = *tslot;

  // ---- the tile's lines into L2 while B is built (one 128 B line per thread, plus the line
  //      holding the last byte of each column piece, whose start is not line-aligned)
  {
    const z32 *piece = nullptr;
    int l = 0, nl = 0;
    if (lower) {                                   // column J + (t >> 3): rows J + jb + m0.., 1 KB
      const int k = t >> 3;
      l = t & 7;
      nl = 8;
      if (k < jb) piece = Am + (size_t)(J + k) * N + (J + jb + m0);
    } else {                                       // column J + jb + m0 + (t >> 2): rows J.., 512 B
      const int cc = t >> 2;
      l = t & 3;
      nl = 4;
      if (cc < nv) piece = Am + (size_t)(J + jb + m0 + cc) * N + J;
    }
    const int bytes = (lower ? nv : jb) * 8;       // valid bytes of the piece
    if (piece && l * 128 < bytes) {
      const char *pc = reinterpret_cast<const char *>(piece);
      asm volatile("prefetch.global.L2 [%0];" ::"l"(pc + l * 128));
      if (l == nl - 1) asm volatile("prefetch.global.L2 [%0];" ::"l"(pc + bytes - 1));
    }
  }

  // ---- B operand: rows n = [Wr(:, n)] (real part of the output), rows 64 + n = [Wi(:, n)]
  //      (imaginary part), hi and lo K blocks; mode 0 W(k, n) = U11^-1(k, n), mode 1
  //      W(k, n) = L11^-1(n, k).  Phase 1 multiplies by [-Wi | Wr]: the same rows with the
  //      halves swapped, the real part's negated (two N = 64 MMAs per slice), so B is built once.
  {
    const int n = t & 63, kq = t >> 6;          // K values kq*8 .. kq*8+7 of column n
    float wr[8], wi[8];
    if (lower) {
      // W(k, n) at W[k + n NB] (NB = 64): staged through the A region (free until the tile's
      // operand is written) so that the global reads are coalesced; 16-byte chunk c of column n
      // (W(2c, n), W(2c + 1, n)) at n * 512 + (c ^ (n & 7)) * 16
      const float4 *w4 = reinterpret_cast<const float4 *>(W);
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int e = t + TT_THREADS * i, wn = e >> 5, c = e & 31;
        *reinterpret_cast<float4 *>(gA + wn * 512 + ((c ^ (wn & 7)) << 4)) = w4[e];
      }
      __syncthreads();
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const float4 v = *reinterpret_cast<const float4 *>(gA + n * 512 + (((4 * kq + j) ^ (n & 7)) << 4));
        wr[2 * j] = v.x;
        wi[2 * j] = v.y;
        wr[2 * j + 1] = v.z;
        wi[2 * j + 1] = v.w;
      }
    } else {
      // W(k, n) at W[k NB + n]: a warp reads 32 consecutive columns
      const z32 *wp = W + kq * 8 * NB + n;
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const z32 w = wp[i * NB];
        wr[i] = w.x;
        wi[i] = w.y;
      }
    }
    put8(gB, n, kq, wr, 1.f);
    put8(gB, 64 + n, kq, wi, 1.f);
    // the staged W is read before the tile's operand overwrites it
    if (lower) __syncthreads();
  }
  asm volatile("" ::: "memory");   // the tile's loads start after it (fewer live registers)

  // ---- the tile, 128 rows x 64 K (zero outside the matrix / beyond jb), loaded once with all of
  //      a thread's loads in flight: real parts feed phase 0, imaginary parts (kept) phase 1;
  //      thread (ar, akq) holds K values akq*16 .. akq*16 + 15 of tile row ar
  float xi[16];
  int ar, akq;
  {
    float xr[16];
    if (lower) {
      // rows J+jb+m0+r, columns J+k: a warp reads 32 consecutive rows of one column
      ar = t & 127;
      akq = t >> 7;
      const z32 *src = Am + (size_t)(J + akq * 16) * N + (J + jb + m0 + ar);
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const int k = akq * 16 + i;
        const z32 v = (ar < nv && k < jb) ? src[i * N] : make_float2(0.f, 0.f);
        xr[i] = v.x;
        xi[i] = v.y;
      }
    } else {
      // columns J+jb+m0+r, rows J+k: four threads per column, 128 contiguous bytes each
      ar = t >> 2;
      akq = t & 3;
      const z32 *src = Am + (size_t)(J + jb + m0 + ar) * N + J;
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int k = akq * 16 + 2 * i;            // jb is even: k, k+1 are both in or both out
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        if (ar < nv && k < jb) v = *reinterpret_cast<const float4 *>(src + k);
        xr[2 * i] = v.x;
        xi[2 * i] = v.y;
        xr[2 * i + 1] = v.z;
        xi[2 * i + 1] = v.w;
      }
    }
#pragma unroll
    for (int q = 0; q < 2; ++q) put8(gA, ar, akq * 2 + q, xr + 8 * q, 1.f);
  }

  // one MMA phase: (hi, hi), (hi, lo), (lo, hi) over the operands in shared memory; phase 0
  // [Cr | Ci] = Xr [Wr | Wi] (N = 128), phase 1 [Cr | Ci] += Xi [-Wi | Wr] (two N = 64 MMAs over
  // B's halves: rows 64.. negated into the real part, rows 0.. into the imaginary part)
  auto mma_phase = [&](int h) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    if (t == 32) {
#pragma unroll
      for (int term = 0; term < 3; ++term)
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const uint32_t a = sA + (term == 2 ? TT_KBLK : 0) + 32 * k;
          const uint32_t bb = sB + (term == 1 ? TT_KBLK : 0) + 32 * k;
          if (h == 0) {
            mma_bf16_tt(tmem, smem_desc(a), smem_desc(bb), IDESC_N128, (term > 0 || k > 0) ? 1u : 0u);
          } else {
            mma_bf16_tt(tmem, smem_desc(a), smem_desc(bb + 64 * 128), IDESC_N64 | (1u << 14), 1u);
            mma_bf16_tt(tmem + 64, smem_desc(a), smem_desc(bb), IDESC_N64, 1u);
          }
        }
      mma_commit(sbar);
    }
  };
  mma_phase(0);
  // the phase-0 MMAs must have read the operands before they are overwritten
  bool ok = __syncthreads_and(mbar_wait(sbar, 0, err, 21));
  if (ok) {
    // ---- A operand of phase 1: the imaginary part of the tile (B stays)
#pragma unroll
    for (int q = 0; q < 2; ++q) put8(gA, ar, akq * 2 + q, xi + 8 * q, 1.f);
    mma_phase(1);
  }
  // CTA-uniform: the epilogue below has block barriers
  if (ok) ok = __syncthreads_and(mbar_wait(sbar, 1, err, 22));
  asm volatile("tcgen05.fence::after_thread_sync;");

  // ---- epilogue: warp w reads TMEM lanes 32 (w % 4).. (tile rows) and output columns
  //      16 (w / 4) .. + 15.  Results reach global memory by TMA stores of four 128 B swizzled
  //      boxes (128 rows x 128 B each) written into the operand region, free once the MMAs
  //      completed: 16-byte piece p of row r of box q at q * 16 KB + r * 128 + (p ^ (r & 7)) * 16
  //      (conflict-free for eight consecutive rows).  Rows and columns outside the matrix or the
  //      staging are clipped by the tensor maps; rows of the tile beyond the panel are zero.
  if (ok) {
    const int quad = warp & 3, grp = warp >> 2;
    const int r = quad * 32 + lane;
    const int n0 = grp * 16;
    unsigned char *box = gA;
    const uint32_t tl = tmem + ((uint32_t)(quad * 32) << 16) + (uint32_t)n0;
    auto sw = [&](int q, int p) { return q * TT_BOX + r * 128 + ((p ^ (r & 7)) << 4); };
    // the thread's 32 output values (16 columns), re then im
    auto tload = [&](float (&re)[16], float (&im)[16]) {
      tmem_ld16(tl, re);
      tmem_ld16(tl + 64, im);
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
    };
    // the four staging segments (pieces n0 / 8 and n0 / 8 + 1 of each 128 B row are this
    // thread's); negb: B's real-part rows [Ur_hi, -Ui_hi, Ur_lo, -Ui_lo], else A's rows
    // [Lr_hi, Li_hi, Lr_lo, Li_lo]
    auto put_stage = [&](const float (&re)[16], const float (&im)[16], bool negb) {
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        const int p = n0 / 8 + c;
        *reinterpret_cast<uint4 *>(box + sw(0, p)) = pack8(re + 8 * c, im + 8 * c, 0, false);
        *reinterpret_cast<uint4 *>(box + sw(1, p)) = pack8(re + 8 * c, im + 8 * c, 2, negb);
        *reinterpret_cast<uint4 *>(box + sw(2, p)) = pack8(re + 8 * c, im + 8 * c, 1, false);
        *reinterpret_cast<uint4 *>(box + sw(3, p)) = pack8(re + 8 * c, im + 8 * c, 3, negb);
      }
    };
    // one thread stores the four boxes: staging rows m0.. (segment q at x = 64 q), or U12 rows
    // J + 16 q.. of columns J + jb + m0..
    auto store_boxes = [&](const CUtensorMap *map, bool fp32_u) {
      fence_async_smem();
      __syncthreads();
      if (t == 0) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          if (fp32_u) tma_store_3d(map, sA + q * TT_BOX, 2 * (J + 16 * q), J + jb + m0, b);
          else tma_store_3d(map, sA + q * TT_BOX, 64 * q, m0, b);
        }
        bulk_commit();
      }
    };
    if (lower) {
      float re[16], im[16];
      tload(re, im);
      // L21 into the matrix (row J+jb+m0+r, columns J+n): a warp stores 32 consecutive rows
      if (r < nv) {
        z32 *dst = Am + (size_t)(J + jb + m0 + r);
#pragma unroll
        for (int j = 0; j < 16; ++j)
          if (n0 + j < jb) dst[(size_t)(J + n0 + j) * N] = make_float2(re[j], im[j]);
      }
      put_stage(re, im, false);
      store_boxes(&maps.stA, false);
    } else {
      {
        // U12 columns: box q holds rows J + 16 q .. + 15 of the tile's 128 columns (row r = column)
        float re[16], im[16];
        tload(re, im);
#pragma unroll
        for (int p = 0; p < 8; ++p)
          *reinterpret_cast<float4 *>(box + sw(grp, p)) =
              make_float4(re[2 * p], im[2 * p], re[2 * p + 1], im[2 * p + 1]);
      }
      store_boxes(&maps.u, true);
      // the boxes are read before the staging overwrites them
      if (t == 0) bulk_wait_read();
      __syncthreads();
      float re[16], im[16];
      tload(re, im);
      put_stage(re, im, true);
      store_boxes(&maps.stB, false);
    }
    // the stores have completed (the next kernels read them) before the CTA leaves
    if (t == 0) bulk_wait_all();
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TT_TMEM_COLS));
  }
}

// ---------------------------------------------------------------------------
// A[b][m][4*NB]: rows m = 0..Mrows-1 are matrix rows J+jb+m, k = 0..NB-1 (zero for k >= jb)
__global__ void __launch_bounds__(256)
k_split_a(const z32 *M, size_t strideM, int N, int J, int jb, int Mrows, int NB, __nv_bfloat16 *A,
          int b0) {
  __shared__ z32 tile[64][65];
  const int b = b0 + blockIdx.y, m0 = blockIdx.x * 64;
  const z32 *L = M + (size_t)b * strideM;
  for (int kc = 0; kc < NB; kc += 64) {
    for (int e = threadIdx.x; e < 64 * 64; e += blockDim.x) {
      int mm = e & 63, kk = e >> 6;
      int m = m0 + mm, k = kc + kk;
      tile[mm][kk] = (m < Mrows && k < jb) ? L[(size_t)(J + jb + m) + (size_t)(J + k) * N]
                                           : make_float2(0.f, 0.f);
    }
    __syncthreads();
    for (int e = threadIdx.x; e < 64 * 64; e += blockDim.x) {
      int kk = e & 63, mm = e >> 6;
      int m = m0 + mm;
      if (m < Mrows) {
        z32 v = tile[mm][kk];
        __nv_bfloat16 rh, rl, ih, il;
        split2(v.x, rh, rl);
        split2(v.y, ih, il);
        __nv_bfloat16 *row = A + ((size_t)b * N + m) * 4 * NB + kc + kk;
        row[0 * NB] = rh; row[1 * NB] = ih;
        row[2 * NB] = rl; row[3 * NB] = il;
      }
    }
    __syncthreads();
  }
}

// B[b][n][4*NB]: the real-part rows [Ur_hi, -Ui_hi, Ur_lo, -Ui_lo] for U rows J..J+jb-1
// and columns n = 0..Ncols-1 (matrix columns J+jb+n); the GEMMs read the imaginary-part
// rows from them (kx_bi, neg_bi)
__global__ void __launch_bounds__(256)
k_split_b(const z32 *M, size_t strideM, int N, int J, int jb, int Ncols, int Ncap, int NB,
          __nv_bfloat16 *B, int b0) {
  const int b = b0 + blockIdx.y;
  const z32 *U = M + (size_t)b * strideM;
  const int n = blockIdx.x * (blockDim.x / NB) + threadIdx.x / NB;
  const int k = threadIdx.x % NB;
  if (n >= Ncols) return;
  z32 v = (k < jb) ? U[(size_t)(J + k) + (size_t)(J + jb + n) * N] : make_float2(0.f, 0.f);
  __nv_bfloat16 rh, rl, ih, il;
  split2(v.x, rh, rl);
  split2(v.y, ih, il);
  __nv_bfloat16 *re = B + ((size_t)b * Ncap + n) * 4 * NB + k;
  re[0 * NB] = rh; re[1 * NB] = __hneg(ih); re[2 * NB] = rl; re[3 * NB] = __hneg(il);
}

// ---------------------------------------------------------------------------
struct TcCtx {
  z32 *M;
  LUBatch lb;
  // operand stagings: set 0 for step-by-step updates, sets 0..G-1 for the steps of a delayed group
  __nv_bfloat16 *A[P_MAXST] = {}, *B[P_MAXST] = {};
  int *err = nullptr;
  int Ncap = 0;
  int nsm = 0;
  bool persist = false;        // C tiles by TMA: needs 16-byte column and matrix strides
  CUtensorMap mapA[P_MAXST], mapB[P_MAXST], mapC;
  CUtensorMap mapC64;          // C halves of 64 rows
  CUtensorMap mapU;            // the matrix as FP32 columns, 128 B swizzled boxes (panel products' stores)
};

bool make_map(CUtensorMap *map, void *base, uint64_t inner, uint64_t rows, uint64_t batch) {
  encode_fn_t enc = tmap_encoder();
  if (!enc) return false;
  cuuint64_t dims[3] = {inner, rows, batch};
  cuuint64_t strides[2] = {inner * 2, inner * rows * 2};
  cuuint32_t box[3] = {BK, 128, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, base, dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

// C as FP32: dims (2N floats per column, columns, matrices), box `rows` rows x 64 columns
bool make_map_c(CUtensorMap *map, void *base, uint64_t N, uint64_t ncols, uint64_t strideM, uint64_t batch,
                uint32_t rows) {
  encode_fn_t enc = tmap_encoder();
  if (!enc) return false;
  cuuint64_t dims[3] = {2 * N, ncols, batch};
  cuuint64_t strides[2] = {N * 8, strideM * 8};
  cuuint32_t box[3] = {2 * rows, P_CH_COLS, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, base, dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

// the matrix as FP32 for the panel products' U12 stores: dims (2N floats per column, columns,
// matrices), box 16 complex rows x 128 columns, 128 B swizzle
bool make_map_u(CUtensorMap *map, void *base, uint64_t N, uint64_t ncols, uint64_t strideM, uint64_t batch) {
  encode_fn_t enc = tmap_encoder();
  if (!enc) return false;
  cuuint64_t dims[3] = {2 * N, ncols, batch};
  cuuint64_t strides[2] = {N * 8, strideM * 8};
  cuuint32_t box[3] = {32, 128, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, base, dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

}  // namespace

int tc_available() {
  int dev = 0, major = 0, minor = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
  cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev);
  return (major == 10 && minor == 0 && tmap_encoder() != nullptr) ? 1 : 0;
}

cudaError_t tc_trail_setup(void **ctx_out, z32 *M, const LUBatch &lb, cudaStream_t st) {
  *ctx_out = nullptr;
  if (lb.NB % 64) return cudaErrorInvalidValue;
  TcCtx *c = new TcCtx();
  c->M = M;
  c->lb = lb;
  c->Ncap = lb.ncols;
  const size_t K4 = 4 * (size_t)lb.NB;       // four staging segments per step
  cudaError_t e = cudaSuccess;
  for (int i = 0; i < P_MAXST && e == cudaSuccess; ++i) {
    e = cudaMalloc(&c->A[i], sizeof(__nv_bfloat16) * K4 * lb.N * lb.batch);
    if (e == cudaSuccess) e = cudaMalloc(&c->B[i], sizeof(__nv_bfloat16) * K4 * c->Ncap * lb.batch);
    if (e == cudaSuccess && (!make_map(&c->mapA[i], c->A[i], K4, lb.N, lb.batch) ||
                             !make_map(&c->mapB[i], c->B[i], K4, (uint64_t)c->Ncap, lb.batch)))
      e = cudaErrorInvalidValue;
  }
  if (e == cudaSuccess) e = cudaMalloc(&c->err, sizeof(int));
  if (e == cudaSuccess) e = cudaMemsetAsync(c->err, 0, sizeof(int), st);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_tc_update, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES);
  // the persistent kernel: C column stride (N * 8 B) and matrix stride on 16 bytes
  if (e == cudaSuccess && lb.N % 2 == 0 && lb.strideM % 2 == 0 &&
      make_map_c(&c->mapC, M, lb.N, lb.ncols, lb.strideM, lb.batch, BM) &&
      make_map_c(&c->mapC64, M, lb.N, lb.ncols, lb.strideM, lb.batch, 64) &&
      make_map_u(&c->mapU, M, lb.N, lb.ncols, lb.strideM, lb.batch) &&
      cudaFuncSetAttribute(k_tc_persist, cudaFuncAttributeMaxDynamicSharedMemorySize, P_SMEM_BYTES) ==
          cudaSuccess) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, dev);
    c->persist = c->nsm > 0;
  }
  if (e != cudaSuccess) {
    for (int i = 0; i < P_MAXST; ++i) { cudaFree(c->A[i]); cudaFree(c->B[i]); }
    cudaFree(c->err);
    delete c;
    return e;
  }
  *ctx_out = c;
  return cudaSuccess;
}

namespace {
// C[crow0 + m, ccol0 + n] -= sum_i A_i.B_i over rows m < Mrows, columns n < Ncols, from the
// stagings i < nst, staging i at row offset ar[i] (A) and column offset bc[i] (B)
cudaError_t persist_region(TcCtx *c, int nst, const int *ar, const int *bc, int first, int count, int crow0,
                           int ccol0, int Mrows, int Ncols, cudaStream_t st) {
  if (Mrows <= 0 || Ncols <= 0 || count <= 0) return cudaSuccess;
  const LUBatch &lb = c->lb;
  const long long ntiles = (long long)cdiv_u(Ncols, BN) * cdiv_u(Mrows, BM) * count;
  const int grid = (int)std::min<long long>(ntiles, c->nsm);
  PMaps maps;
  POff off{};
  for (int i = 0; i < P_MAXST; ++i) {
    maps.a[i] = c->mapA[i];
    maps.b[i] = c->mapB[i];
    off.ar[i] = i < nst ? ar[i] : 0;
    off.bc[i] = i < nst ? bc[i] : 0;
  }
  maps.c = c->mapC;
  maps.c64 = c->mapC64;
  k_tc_persist<<<grid, P_THREADS, P_SMEM_BYTES, st>>>(maps, c->M, lb.strideM, lb.N, crow0, ccol0, off, nst,
                                                       lb.NB / BK, Mrows, Ncols, first, count, c->err);
  return ADGA_LAUNCH_CHECK();
}

// staging of one step: L rows J + jb.., columns J..J + jb; U rows J..J + jb, columns J + jb..
cudaError_t stage_step(TcCtx *c, __nv_bfloat16 *A, __nv_bfloat16 *B, int first, int count, int J, int jb,
                       cudaStream_t st) {
  const LUBatch &lb = c->lb;
  const int Mrows = lb.N - J - jb, Ncols = lb.ncols - J - jb, NB = lb.NB;
  if (Mrows > 0) {
    k_split_a<<<dim3(cdiv_u(Mrows, 64), count), 256, 0, st>>>(c->M, lb.strideM, lb.N, J, jb, Mrows, NB, A, first);
    cudaError_t e = ADGA_LAUNCH_CHECK();
    if (e != cudaSuccess) return e;
  }
  if (Ncols > 0) {
    k_split_b<<<dim3(cdiv_u(Ncols, 256 / NB), count), 256, 0, st>>>(c->M, lb.strideM, lb.N, J, jb, Ncols, c->Ncap,
                                                                     NB, B, first);
    return ADGA_LAUNCH_CHECK();
  }
  return cudaSuccess;
}
}  // namespace

cudaError_t tc_trail_run_range(void *ctxp, int first, int count, int J, int jb, cudaStream_t st,
                               cudaEvent_t ev0, cudaEvent_t ev1) {
  TcCtx *c = (TcCtx *)ctxp;
  const LUBatch &lb = c->lb;
  const int Mrows = lb.N - J - jb, Ncols = lb.ncols - J - jb;
  if (Mrows <= 0 || Ncols <= 0 || count <= 0) return cudaSuccess;
  const int NB = lb.NB;
  cudaError_t e = stage_step(c, c->A[0], c->B[0], first, count, J, jb, st);
  if (e != cudaSuccess) return e;
  if (ev0) cudaEventRecord(ev0, st);
  if (c->persist) {
    const int zero[1] = {0};
    e = persist_region(c, 1, zero, zero, first, count, J + jb, J + jb, Mrows, Ncols, st);
  } else {
    dim3 grid(cdiv_u(Ncols, BN), cdiv_u(Mrows, BM), count);
    k_tc_update<<<grid, 192, SMEM_BYTES, st>>>(c->mapA[0], c->mapB[0], c->M, lb.strideM, lb.N, J, jb, Mrows, Ncols,
                                               c->Ncap, 6 * NB / BK, first, NB / BK, c->err);
    e = ADGA_LAUNCH_CHECK();
  }
  if (ev1) cudaEventRecord(ev1, st);
  return e;
}

// ---------------------------------------------------------------------------
// Delayed updates of the unpivoted path in groups of G steps (G = 2..4): after step
// g of a group (steps J_i, widths jb_i, i <= g, staged in sets i):
//   g < G - 1   the group's updates so far restricted to what step g + 1 reads: its
//               columns below it and its rows right of it (K = (g + 1) * 6 NB);
//   g = G - 1   the rest, rows and columns from J_g + jb_g, with all G steps' L21 / U12
//               as one K = G * 6 NB product.
// The C read-modify-write of the largest region happens once per G steps.
// ---------------------------------------------------------------------------
int tc_pair_supported(void *ctxp) { return ctxp && ((TcCtx *)ctxp)->persist && ((TcCtx *)ctxp)->lb.NB == 64; }

cudaError_t tc_group_update(void *ctxp, int first, int count, int nst, const int *Js, const int *jbs, bool wide,
                            cudaStream_t st, cudaEvent_t ev0, cudaEvent_t ev1, bool staged) {
  TcCtx *c = (TcCtx *)ctxp;
  const LUBatch &lb = c->lb;
  if (nst < 1 || nst > P_MAXST) return cudaErrorInvalidValue;
  const int g = nst - 1;
  cudaError_t e = staged ? cudaSuccess : stage_step(c, c->A[g], c->B[g], first, count, Js[g], jbs[g], st);
  if (e != cudaSuccess) return e;
  const int R = Js[g] + jbs[g];             // first row / column after the newest step
  int ar[P_MAXST], bc[P_MAXST];
  auto offsets = [&](int crow0, int ccol0) {
    for (int i = 0; i < nst; ++i) {
      ar[i] = crow0 - (Js[i] + jbs[i]);
      bc[i] = ccol0 - (Js[i] + jbs[i]);
    }
  };
  if (ev0) cudaEventRecord(ev0, st);
  if (wide) {
    offsets(R, R);
    e = persist_region(c, nst, ar, bc, first, count, R, R, lb.N - R, lb.ncols - R, st);
  } else {
    const int jt = std::min(lb.NB, lb.N - R);   // the next step's width
    // its columns, every row below R
    offsets(R, R);
    e = persist_region(c, nst, ar, bc, first, count, R, R, lb.N - R, jt, st);
    // its rows, the columns right of it
    if (e == cudaSuccess) {
      offsets(R, R + jt);
      e = persist_region(c, nst, ar, bc, first, count, R, R + jt, jt, lb.ncols - R - jt, st);
    }
  }
  if (ev1) cudaEventRecord(ev1, st);
  return e;
}

// L21 and U12 of unpivoted step (J, jb) on the tensor cores (k_tc_tri), which also
// writes the step's operand staging set (its index in its delayed group)
cudaError_t tc_tri_step(void *ctxp, int first, int count, int J, int jb, int set, cudaStream_t st) {
  TcCtx *c = (TcCtx *)ctxp;
  const LUBatch &lb = c->lb;
  if (!c->persist || lb.NB != 64 || (jb & 1) || set < 0 || set >= P_MAXST) return cudaErrorInvalidValue;
  const int ntA = (int)cdiv_u(std::max(lb.N - J - jb, 0), TT_ROWS);
  const int ntU = (int)cdiv_u(std::max(lb.ncols - J - jb, 0), TT_ROWS);
  if (ntA + ntU == 0 || count <= 0) return cudaSuccess;
  cudaError_t e = smem_limit(k_tc_tri, TT_SMEM_BYTES);
  if (e != cudaSuccess) return e;
  TriMaps maps;
  maps.stA = c->mapA[set];
  maps.stB = c->mapB[set];
  maps.u = c->mapU;
  k_tc_tri<<<(unsigned)((ntA + ntU) * count), TT_THREADS, TT_SMEM_BYTES, st>>>(
      maps, c->M, lb.strideM, lb.N, lb.ncols, J, jb, lb.NB, lb.nsteps(), (const z32 *)lb.Linv,
      (const z32 *)lb.Uinv, first, ntA, ntU, c->err);
  return ADGA_LAUNCH_CHECK();
}

int tc_trail_error(void *ctxp) {
  TcCtx *c = (TcCtx *)ctxp;
  int v = 0;
  if (cudaMemcpy(&v, c->err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
  return v;
}

// the device flag the tensor-core kernels' bounded waits report to
int *tc_err_flag(void *ctxp) { return ctxp ? ((TcCtx *)ctxp)->err : nullptr; }

void tc_trail_free(void *ctxp) {
  TcCtx *c = (TcCtx *)ctxp;
  if (!c) return;
  for (int i = 0; i < P_MAXST; ++i) {
    cudaFree(c->A[i]);
    cudaFree(c->B[i]);
  }
  cudaFree(c->err);
  delete c;
}
