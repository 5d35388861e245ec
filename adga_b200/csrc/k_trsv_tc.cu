// Triangular solves of the mixed path on the tensor cores: U X = Y and the
// unit-lower L Y = B of the FP32 factors without row interchanges, for
// R <= 16 right-hand sides (the BSE's ndim^2 columns; the FP64 path and the
// pivoted FP32 factors keep the streaming solves of k_trsv.cu).
//
// Right-looking blocked solve, one CTA per matrix.  Once block p (64 rows) is
// solved, the rows still to solve are updated, B[rows] -= T[rows, block p] Y_p,
// on the tensor cores, and every row block keeps its accumulated update in
// TMEM for the whole solve:
//   * the triangle's tiles (64 complex rows x 32 columns of one panel, 16 KB
//     FP32) stream through a 5-stage TMA ring as they lie in memory, real
//     and imaginary parts interleaved;
//   * warps 4-7 split every landed tile into hi = tf32(x) (round to nearest)
//     and lo = x - hi (exact in FP32) and write both as the K-major A
//     operand of an M = 128 MMA whose rows are the real and imaginary parts
//     of the 64 complex rows (kind::tf32, N = 32, K = 8 per instruction);
//     the ring slot is free again once read, the operand pair once its MMAs
//     complete (two pairs);
//   * the B operand holds Y_p's real parts (rows 0..15) and imaginary parts
//     (16..31), so TMEM lane 2r accumulates [Tr Yr | Tr Yi] and lane 2r + 1
//     [Ti Yr | Ti Yi] of complex row r; the complex update is the
//     combination across the lane pair (Tr Yr - Ti Yi, Tr Yi + Ti Yr);
//   * three-term TF32 products hi*hi + hi*lo + lo*hi, about 2^-21 relative
//     per product, FP32 accumulation;
//   * warp 0 issues the TMA loads, warp 1 the MMAs (one thread each), warps
//     8-11 solve the diagonal blocks, Y_p = D_p^-1 (B_p - acc_p) with the
//     64 x 64 block inverses of k_diag_inv, as soon as the first tile of the
//     previous panel (the one that updates block p) has completed, so that
//     the rest of that panel streams meanwhile.
// TMEM holds one 32-column accumulator per row block after the first solved
// one: N <= 17 * 64 = 1088.  Every wait is bounded (WAIT_NS); on a timeout the
// kernel records an error code in *err and returns.
//
// The reference solves nothing itself: it inverts with zgetrf + zgetri
// (src/lapack_module.f90:40-70); the mixed path's solves replace the
// triangular-solve part of that inversion.
#include "lu.cuh"
#include "umma.cuh"
#include <cuda.h>

namespace {

using namespace umma;

constexpr int QB = 64;                        // block width (the factorisation's NB)
constexpr int Q_THREADS = 384;
constexpr int Q_NS = 5;                       // ring stages
constexpr int Q_KC = 32;                      // panel columns per stage
constexpr int Q_STAGE = 128 * Q_KC * 4;       // 128 reals (64 complex rows) x 32 columns FP32 (16 KB)
constexpr int Q_NP = 32;                      // MMA N: 16 real-part + 16 imaginary-part rows of B
constexpr int Q_RMAX = 16;
constexpr int Q_BOP = Q_NP * QB * 4;          // one B operand (hi or lo): 32 rows x 64 K, tf32 (8 KB)
constexpr int Q_DINV = QB * QB * 8;           // one block inverse, FP32 complex (32 KB)
constexpr int Q_VST = QB * Q_RMAX * 8;        // B_p - acc_p, [rhs][row] complex (8 KB)
constexpr int Q_MAXBLK = 17;                  // TMEM: (blocks - 1) x 32 columns <= 512
constexpr int OFF_RING = 0;
constexpr int OFF_AOP = OFF_RING + Q_NS * Q_STAGE;   // two A operand pairs (hi, lo), K-major
constexpr int OFF_BOP = OFF_AOP + 4 * Q_STAGE;       // two B operand pairs (hi, lo)
constexpr int OFF_DINV = OFF_BOP + 4 * Q_BOP;
constexpr int OFF_VST = OFF_DINV + Q_DINV;
constexpr int OFF_BAR = OFF_VST + Q_VST;
// full[NS] empty[NS] conv[2] opfree[2] crit yready dfull done
constexpr int Q_NBAR = 2 * Q_NS + 8;
constexpr int Q_SMEM = OFF_BAR + 8 * Q_NBAR + 16 + 1024;
static_assert(Q_SMEM <= 227 * 1024, "shared memory of the tensor-core solve");

// kind::tf32, D = F32, A and B K-major, M = 128, N = 32
constexpr uint32_t IDESC_TF32 = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(Q_NP / 8) << 17) |
                                ((uint32_t)(128 / 16) << 24);

// K-major, 128 B swizzle: LBO unused, SBO = 1 KB between 8-row groups
__device__ __forceinline__ uint64_t desc_k(uint32_t addr) {
  uint64_t d = 0;
  d |= (uint64_t)((addr & 0x3FFFF) >> 4);
  d |= (uint64_t)1 << 16;
  d |= (uint64_t)(1024 >> 4) << 32;
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)2 << 61;
  return d;
}
__device__ __forceinline__ void mma_tf32(uint32_t tmem, uint64_t a, uint64_t b, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
      "l"(a), "l"(b), "r"(IDESC_TF32), "r"(acc));
}
// x rounded to the nearest TF32 (low 13 mantissa bits zero)
__device__ __forceinline__ float tf32_rna(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}
// byte offset of element (m, k) of a K-major A operand: 128 rows, K = 32 (one 128 B row each)
__device__ __forceinline__ uint32_t aop_off(int m, int k) {
  return (uint32_t)((m >> 3) * 1024 + (m & 7) * 128 + (((k >> 2) ^ (m & 7)) << 4) + (k & 3) * 4);
}
// byte offset of element (n, k) of a K-major B operand: 32 rows, K = 64 as two 128 B atoms
__device__ __forceinline__ uint32_t bop_off(int n, int k) {
  return (uint32_t)((k >> 5) * 4096 + (n >> 3) * 1024 + (n & 7) * 128 + ((((k & 31) >> 2) ^ (n & 7)) << 4) +
                    (k & 3) * 4);
}
__device__ __forceinline__ void bulk_load(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}
__device__ __forceinline__ void named_sync(int id, int n) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory");
}
// named barrier that also ANDs a flag over its threads (so that they take the same branch after it)
__device__ __forceinline__ bool named_and(int id, int n, bool v) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.b32 p, %1, 0;\n\t"
      "bar.red.and.pred q, %2, %3, p;\n\t"
      "selp.b32 %0, 1, 0, q;\n\t}"
      : "=r"(r)
      : "r"((int)v), "r"(id), "r"(n)
      : "memory");
  return r != 0;
}

// Solve order: position p -> block index; panel p (the solved block p) updates
// ntiles(p) blocks, the next one to solve first.
struct QGeo {
  int nblk;
  bool upper;
  __device__ int blk(int p) const { return upper ? nblk - 1 - p : p; }
  __device__ int ntiles(int p) const { return nblk - 1 - p; }
  __device__ int tile_blk(int p, int t) const { return upper ? nblk - 2 - p - t : p + 1 + t; }
  __device__ uint32_t tcol(int j) const { return (uint32_t)((upper ? j : j - 1) * Q_NP); }
};

__global__ void __launch_bounds__(Q_THREADS, 1)
k_trsv_tc(const __grid_constant__ CUtensorMap tmap, int N, int nsteps, const z32 *__restrict__ Dinv, z32 *C,
          size_t strideC, int ldc, int R, int upper_i, int *err) {
  extern __shared__ unsigned char smraw[];
  const uint32_t s0 = (smem_u32(smraw) + 1023u) & ~1023u;
  unsigned char *g0 = smraw + (s0 - smem_u32(smraw));
  const uint32_t bar0 = s0 + OFF_BAR;
  const uint32_t b_full = bar0, b_empty = bar0 + 8 * Q_NS, b_conv = bar0 + 16 * Q_NS, b_opfree = b_conv + 16;
  const uint32_t b_crit = b_opfree + 16, b_yready = b_crit + 8, b_dfull = b_crit + 16, b_done = b_crit + 24;
  uint32_t *tslot = reinterpret_cast<uint32_t *>(g0 + OFF_BAR + 8 * Q_NBAR);
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const int b = blockIdx.x;
  const QGeo geo{(N + QB - 1) / QB, upper_i != 0};
  const int nblk = geo.nblk;
  z32 *Cb = C + (size_t)b * strideC;
  const z32 *Db = Dinv + (size_t)b * nsteps * QB * QB;

  if (t == 0) {
    for (int s = 0; s < Q_NS; ++s) {
      mbar_init(b_full + 8 * s, 1);
      mbar_init(b_empty + 8 * s, 128);
    }
    for (int i = 0; i < 2; ++i) {
      mbar_init(b_conv + 8 * i, 128);
      mbar_init(b_opfree + 8 * i, 1);
    }
    for (int i = 0; i < 4; ++i) mbar_init(b_crit + 8 * i, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  // both B operand sets start at zero: rows n >= R (and 16 + n) are never written
  for (int e = t; e < 4 * Q_BOP / 16; e += Q_THREADS)
    reinterpret_cast<uint4 *>(g0 + OFF_BOP)[e] = make_uint4(0u, 0u, 0u, 0u);
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                 "r"(512));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = *tslot;

  if (warp == 0) {
    // ---- TMA producer: the stages of every panel in solve order
    if (lane == 0) {
      bool ok = true;
      int g = 0;
      for (int p = 0; p < nblk - 1 && ok; ++p) {
        const int col0 = geo.blk(p) * QB;
        for (int tt = 0; tt < geo.ntiles(p) && ok; ++tt) {
          const int j = geo.tile_blk(p, tt);
          for (int h = 0; h < 2; ++h, ++g) {
            const int s = g % Q_NS;
            if (g >= Q_NS && !(ok = mbar_wait(b_empty + 8 * s, ((g / Q_NS) - 1) & 1, err, 41))) break;
            mbar_expect_tx(b_full + 8 * s, Q_STAGE);
            tma_load_3d(s0 + OFF_RING + s * Q_STAGE, &tmap, b_full + 8 * s, 128 * j, col0 + Q_KC * h, b);
          }
        }
      }
    }
  } else if (warp == 1) {
    // ---- MMA issuer
    if (lane == 0 && nblk > 1) {
      bool ok = true;
      int g = 0;
      for (int p = 0; p < nblk - 1 && ok; ++p) {
        if (!(ok = mbar_wait(b_yready, p & 1, err, 42))) break;
        asm volatile("tcgen05.fence::after_thread_sync;");
        const uint32_t bop = s0 + OFF_BOP + (p & 1) * 2 * Q_BOP;
        for (int tt = 0; tt < geo.ntiles(p) && ok; ++tt) {
          const uint32_t dt = tmem + geo.tcol(geo.tile_blk(p, tt));
          for (int h = 0; h < 2; ++h, ++g) {
            const int o = g & 1;
            if (!(ok = mbar_wait(b_conv + 8 * o, (g >> 1) & 1, err, 43))) break;
            asm volatile("tcgen05.fence::after_thread_sync;");
            const uint32_t ahi = s0 + OFF_AOP + o * 2 * Q_STAGE, alo = ahi + Q_STAGE;
#pragma unroll
            for (int term = 0; term < 3; ++term)
#pragma unroll
              for (int k = 0; k < 4; ++k) {
                const uint32_t a = (term == 2 ? alo : ahi) + 32 * k;
                const uint32_t bb = bop + (term == 1 ? Q_BOP : 0) + 4096 * h + 32 * k;
                mma_tf32(dt, desc_k(a), desc_k(bb), (p > 0 || h > 0 || term > 0 || k > 0) ? 1u : 0u);
              }
            mma_commit(b_opfree + 8 * o);
            if (tt == 0 && h == 1) mma_commit(b_crit);
          }
        }
      }
      mma_commit(b_done);
      mbar_wait(b_done, 0, err, 48);
    }
  } else if (warp >= 4 && warp < 8) {
    // ---- every landed tile (128 reals x 32 columns, as loaded) into the K-major A operand pair:
    //      thread m owns row m (real index 128 j + m), hi = tf32(x), lo = x - hi
    const int m = t - 128;
    bool ok = true;
    int g = 0;
    for (int p = 0; p < nblk - 1 && ok; ++p)
      for (int tt = 0; tt < geo.ntiles(p) && ok; ++tt)
        for (int h = 0; h < 2; ++h, ++g) {
          const int s = g % Q_NS, o = g & 1;
          ok = mbar_wait(b_full + 8 * s, (g / Q_NS) & 1, err, 44);
          if (ok && g >= 2) ok = mbar_wait(b_opfree + 8 * o, ((g >> 1) - 1) & 1, err, 45);
          if (!ok) break;
          const float *src = reinterpret_cast<const float *>(g0 + OFF_RING + s * Q_STAGE);
          float x[Q_KC];
#pragma unroll
          for (int k = 0; k < Q_KC; ++k) x[k] = src[k * 128 + m];
          // the ring slot is read: the next load may land there
          mbar_arrive(b_empty + 8 * s);
          unsigned char *ahi = g0 + OFF_AOP + o * 2 * Q_STAGE, *alo = ahi + Q_STAGE;
#pragma unroll
          for (int k = 0; k < Q_KC; k += 4) {
            const float4 hv = make_float4(tf32_rna(x[k]), tf32_rna(x[k + 1]), tf32_rna(x[k + 2]), tf32_rna(x[k + 3]));
            *reinterpret_cast<float4 *>(ahi + aop_off(m, k)) = hv;
            *reinterpret_cast<float4 *>(alo + aop_off(m, k)) =
                make_float4(x[k] - hv.x, x[k + 1] - hv.y, x[k + 2] - hv.z, x[k + 3] - hv.w);
          }
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
          mbar_arrive(b_conv + 8 * o);
        }
  } else if (warp >= 8) {
    // ---- diagonal blocks: Y_p = D_p^-1 (B_p - acc_p)
    const int dt_ = t - 256, q = warp & 3;
    float2 *vst = reinterpret_cast<float2 *>(g0 + OFF_VST);   // [rhs][row]
    const float2 *D = reinterpret_cast<const float2 *>(g0 + OFF_DINV);
    if (dt_ == 0) {
      mbar_expect_tx(b_dfull, Q_DINV);
      bulk_load(s0 + OFF_DINV, Db + (size_t)geo.blk(0) * QB * QB, Q_DINV, b_dfull);
    }
    for (int p = 0; p < nblk; ++p) {
      const int r0 = geo.blk(p) * QB, jb = min(QB, N - r0);
      // this lane's right-hand-side values of block p (row r, part c), loaded before the wait for
      // the accumulator so that their latency overlaps it
      const int r = q * 16 + (lane >> 1), c = lane & 1;
      float bv[Q_RMAX];
#pragma unroll
      for (int n = 0; n < Q_RMAX; ++n) {
        bv[n] = 0.f;
        if (p > 0 && n < R && r < jb) bv[n] = reinterpret_cast<const float *>(Cb + (size_t)(r0 + r) + (size_t)n * ldc)[c];
      }
      bool w = true;
      if (p > 0) w = mbar_wait(b_crit, (p - 1) & 1, err, 46);
      w = w && mbar_wait(b_dfull, p & 1, err, 47);
      if (!named_and(1, 128, w)) break;
      if (p > 0) {
        asm volatile("tcgen05.fence::after_thread_sync;");
        float v[32];
        const uint32_t ta = tmem + ((uint32_t)(q * 32) << 16) + geo.tcol(geo.blk(p));
        tmem_ld16(ta, *reinterpret_cast<float(*)[16]>(v));
        tmem_ld16(ta + 16, *reinterpret_cast<float(*)[16]>(v + 16));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        // lane 2r: [Tr Yr | Tr Yi], lane 2r + 1: [Ti Yr | Ti Yi] of complex row r
#pragma unroll
        for (int n = 0; n < Q_RMAX; ++n) {
          const float pv = __shfl_xor_sync(0xffffffffu, v[16 + n], 1);
          const float upd = c ? v[n] + pv : v[n] - pv;
          if (n < R) reinterpret_cast<float *>(vst)[(n * QB + r) * 2 + c] = r < jb ? bv[n] - upd : 0.f;
        }
      } else {
        for (int e = dt_; e < QB * R; e += 128) {
          const int r = e % QB, n = e / QB;
          vst[n * QB + r] = r < jb ? Cb[(size_t)(r0 + r) + (size_t)n * ldc] : make_float2(0.f, 0.f);
        }
      }
      named_sync(1, 128);
      unsigned char *bh = g0 + OFF_BOP + (p & 1) * 2 * Q_BOP, *bl = bh + Q_BOP;
      for (int e = dt_; e < QB * R; e += 128) {
        const int r = e % QB, n = e / QB;
        z32 y = make_float2(0.f, 0.f);
        if (r < jb) {
          // D^-1 of U is upper triangular, of the unit-lower L lower triangular
          const int kb = geo.upper ? r : 0, ke = geo.upper ? jb : r + 1;
          const float2 *vn = vst + n * QB;
          z32 a0 = make_float2(0.f, 0.f), a1 = make_float2(0.f, 0.f);
          int k = kb;
          for (; k + 1 < ke; k += 2) {
            cfma(a0, D[r + k * QB], vn[k]);
            cfma(a1, D[r + (k + 1) * QB], vn[k + 1]);
          }
          if (k < ke) cfma(a0, D[r + k * QB], vn[k]);
          y = cadd(a0, a1);
          Cb[(size_t)(r0 + r) + (size_t)n * ldc] = y;
        }
        const float hr = tf32_rna(y.x), hi = tf32_rna(y.y);
        *reinterpret_cast<float *>(bh + bop_off(n, r)) = hr;
        *reinterpret_cast<float *>(bl + bop_off(n, r)) = y.x - hr;
        *reinterpret_cast<float *>(bh + bop_off(16 + n, r)) = hi;
        *reinterpret_cast<float *>(bl + bop_off(16 + n, r)) = y.y - hi;
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      named_sync(1, 128);
      if (dt_ == 0) {
        mbar_arrive(b_yready);
        // the next block inverse into the buffer just read
        if (p + 1 < nblk) {
          mbar_expect_tx(b_dfull, Q_DINV);
          bulk_load(s0 + OFF_DINV, Db + (size_t)geo.blk(p + 1) * QB * QB, Q_DINV, b_dfull);
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512));
  }
}

}  // namespace

bool trsv_tc_supported(const LUBatch &lb, int R, bool upper) {
  return lb.tc_err && lb.NB == QB && R >= 1 && R <= Q_RMAX && (lb.N + QB - 1) / QB <= Q_MAXBLK && lb.N % 2 == 0 &&
         lb.strideM % 2 == 0 && (upper || lb.nopiv) && tmap_encoder() != nullptr;
}

cudaError_t launch_trsv_tc(const z32 *M, const LUBatch &lb, z32 *C, size_t strideC, int ldc, int R, bool upper,
                           cudaStream_t st) {
  // the factors as FP32: (2N reals of a column, N columns, matrices); the right-hand
  // sides stored beside them (columns N..) lie outside the map and read as zeros
  CUtensorMap map;
  cuuint64_t dims[3] = {2 * (cuuint64_t)lb.N, (cuuint64_t)lb.N, (cuuint64_t)lb.batch};
  cuuint64_t strides[2] = {(cuuint64_t)lb.N * 8, (cuuint64_t)lb.strideM * 8};
  cuuint32_t box[3] = {128, Q_KC, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  if (tmap_encoder()(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<z32 *>(M), dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return cudaErrorInvalidValue;
  cudaError_t e = smem_limit(k_trsv_tc, Q_SMEM);
  if (e != cudaSuccess) return e;
  k_trsv_tc<<<lb.batch, Q_THREADS, Q_SMEM, st>>>(map, lb.N, lb.nsteps(), (const z32 *)(upper ? lb.Uinv : lb.Linv),
                                                 C, strideC, ldc, R, upper ? 1 : 0, lb.tc_err);
  return ADGA_LAUNCH_CHECK();
}
