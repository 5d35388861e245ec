// FP64-accurate refinement residual of the mixed path on the int8 tensor cores.
//
// The residual r = B - X + (X D) F~ (k_refine.cu) needs the product P = XD F~
// to ~1e-13 relative accuracy.  Here P is formed exactly from integer slices
// (the Ozaki splitting, with an exact integer accumulation) instead of FP64
// FMAs:
//   * the complex product runs as one real product of the embeddings
//         A = [Re XD | Im XD]                       (rows p,i1 ; K2 = 2N)
//         B(c re) = [Re F~(:,c) ; -Im F~(:,c)],  B(c im) = [Im F~(:,c) ; Re F~(:,c)];
//   * every row of A and every column c of F~ is scaled by a power of two,
//     v = 2^e u with |u| < 1, and u is cut into S = 7 signed digits of base
//     2^7 by rounding, u = sum_p d_p 2^(1 - 7p), |d_p| <= 64 (exact in FP64);
//   * the slice products sum_k dA_p dB_q (|.| <= 64*64*K2) are exact in int32;
//     the 28 pairs with p + q <= S + 1 are grouped by g = p + q, each group in
//     its own TMEM accumulator (7 x 64 columns), and
//         P = 2^(eA + eB + 2) sum_g 2^(-7 g) G_g
//     is assembled in FP64 in the epilogue (error ~2^-49 of the row / column
//     scales; the dropped pairs are below it).
// The GEMM (k_resid_i8): one CTA per 128-row x 64-real-column tile
// (32 complex columns), K in 64-byte chunks through a 2-stage TMA ring (all
// seven A and seven B slices of a chunk per stage, 84 KB, SWIZZLE_64B, no
// multicast), tcgen05.mma.kind::i8 (M = 128, N = 64, K = 32) issued by one
// thread, and eight epilogue warps that combine the groups, form r, store it
// as FP32 for the correction solve and record max|r| per matrix (as
// k_resid_z64 does).  Every mbarrier wait is bounded.
// The slices of F~ depend on omega only and are cut once per omega slice.
#include "ctx.cuh"
#include "umma.cuh"
#include <cuda.h>
#include <algorithm>

namespace {

using namespace umma;

constexpr int S = 7;                 // digits per value
constexpr int NG = S;                // groups g = p + q = 2 .. S + 1
constexpr int RB_M = 128;            // tile rows
constexpr int RB_N = 64;             // tile real columns (32 complex)
constexpr int KC = 64;               // K bytes per stage (one 64 B swizzle row)
constexpr int A_SL = RB_M * KC;      // 8 KB: one A slice of a chunk
constexpr int B_SL = RB_N * KC;      // 4 KB: one B slice of a chunk
constexpr int STG = S * (A_SL + B_SL);   // 84 KB per stage
constexpr int NSTG = 2;
constexpr int RI_THREADS = 384;
constexpr int RI_SMEM = NSTG * STG + 1024 + 256;
constexpr int TMEM_COLS = 512;       // NG x 64 = 448 used

// K-major, 64 B swizzle: SBO = 512 B between 8-row groups
__device__ __forceinline__ uint64_t desc_sw64(uint32_t addr) {
  uint64_t d = 0;
  d |= (uint64_t)((addr & 0x3FFFF) >> 4);
  d |= (uint64_t)1 << 16;                 // leading byte offset (unused for swizzled K-major)
  d |= (uint64_t)(512 >> 4) << 32;        // stride byte offset
  d |= (uint64_t)1 << 46;                 // descriptor version (sm_100)
  d |= (uint64_t)4 << 61;                 // SWIZZLE_64B
  return d;
}
// kind::i8, A = B = S8, D = S32, both K-major, M = 128, N = 64
constexpr uint32_t IDESC_I8 = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(RB_N / 8) << 17) |
                              ((uint32_t)(RB_M / 16) << 24);
__device__ __forceinline__ void mma_i8(uint32_t tmem, uint64_t a, uint64_t b, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
      "l"(a), "l"(b), "r"(IDESC_I8), "r"(acc));
}
__device__ __forceinline__ void tmem_ld16i(uint32_t taddr, int (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = (int)r[i];
}

// exponent e with |v| < 2^e for every |v| <= m (0 for m = 0)
__device__ __forceinline__ int scale_exp(double m) {
  int e = 0;
  if (m > 0.0) frexp(m, &e);
  return e;
}
// the S digits of u (|u| < 1): u = sum_p d_p 2^(1 - 7p)
__device__ __forceinline__ void digits(double u, signed char (&d)[S]) {
  double x = u * 64.0;
#pragma unroll
  for (int p = 0; p < S; ++p) {
    const double r = rint(x);
    d[p] = (signed char)r;
    x = (x - r) * 128.0;
  }
}

// Slices of XD for channel ch: one warp per row (p, i1); A value kk of the row
// is Re XD(kk) for kk < N, Im XD(kk - N) below 2N, zero up to K2p.
__global__ void __launch_bounds__(256)
k_slice_rows(int N, int R, int npts, int ch, const z64 *__restrict__ XD, signed char *__restrict__ As,
             int *__restrict__ eA, int K2p, size_t rows_cap) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  const int rows = npts * R;
  if (warp >= rows) return;
  const int p = warp / R, i1 = warp % R;
  const z64 *x = XD + (size_t)(2 * p + ch) * R * N + (size_t)i1 * N;
  double m = 0.0;
  for (int k = lane; k < N; k += 32) m = fmax(m, fmax(fabs(x[k].x), fabs(x[k].y)));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  const int e = scale_exp(m);
  if (lane == 0) eA[(size_t)ch * rows_cap + warp] = e;
  for (int kk = lane; kk < K2p; kk += 32) {
    double v = 0.0;
    if (kk < N) v = x[kk].x;
    else if (kk < 2 * N) v = x[kk - N].y;
    signed char d[S];
    digits(ldexp(v, -e), d);
#pragma unroll
    for (int q = 0; q < S; ++q) As[((size_t)(ch * S + q) * rows_cap + warp) * K2p + kk] = d[q];
  }
}

// Slices of F~ (row-major, F~(k, c) at Frow[k N + c]) for channel ch.  B row rb in
// tile order: tile rb / 64, j = rb % 64, complex column c = 32 tile + j % 32, part
// j / 32 (0: [Re F~(:,c) ; -Im F~(:,c)], 1: [Im F~(:,c) ; Re F~(:,c)]).  One warp per B row.
__global__ void __launch_bounds__(256)
k_slice_cols(int N, int ch, const z64 *__restrict__ Frow, signed char *__restrict__ Bs, int *__restrict__ eB,
             int K2p, int N2p) {
  const int rb = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (rb >= N2p) return;
  const int j = rb % RB_N, c = (rb / RB_N) * (RB_N / 2) + (j % (RB_N / 2)), part = j / (RB_N / 2);
  const bool cv = c < N;
  double m = 0.0;
  if (cv)
    for (int k = lane; k < N; k += 32) {
      const z64 f = Frow[(size_t)k * N + c];
      m = fmax(m, fmax(fabs(f.x), fabs(f.y)));
    }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  const int e = scale_exp(m);
  if (lane == 0 && part == 0 && cv) eB[(size_t)ch * N + c] = e;
  for (int kk = lane; kk < K2p; kk += 32) {
    double v = 0.0;
    if (cv && kk < 2 * N) {
      const z64 f = Frow[(size_t)(kk < N ? kk : kk - N) * N + c];
      v = part == 0 ? (kk < N ? f.x : -f.y) : (kk < N ? f.y : f.x);
    }
    signed char d[S];
    digits(ldexp(v, -e), d);
#pragma unroll
    for (int q = 0; q < S; ++q) Bs[((size_t)(ch * S + q) * N2p + rb) * K2p + kk] = d[q];
  }
}

// The residual GEMM and its epilogue for channel ch (see the file comment).
//   warp 0: TMA loads of the 14 slices of each K chunk; warp 1: TMEM allocation and the
//   MMAs; warps 4..11: epilogue (warp w: TMEM lanes 32 (w % 4).., complex columns
//   16 ((w - 4) / 4) .. + 15 of the tile).
__global__ void __launch_bounds__(RI_THREADS, 1)
k_resid_i8(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB, int N, int R,
           int npts, int ch, int nkc, const int *__restrict__ eA, const int *__restrict__ eB, size_t rows_cap,
           const z64 *__restrict__ X, const z64 *__restrict__ opg, z32 *V, const z64 *__restrict__ extra,
           unsigned long long *rnorm, const z64 *__restrict__ Bpt, int *err) {
  extern __shared__ unsigned char smraw[];
  const uint32_t sbase = (smem_u32(smraw) + 1023u) & ~1023u;
  unsigned char *g = smraw + (sbase - smem_u32(smraw));
  uint64_t *bars = reinterpret_cast<uint64_t *>(g + NSTG * STG);
  uint32_t *tslot = reinterpret_cast<uint32_t *>(bars + 2 * NSTG + 1);
  const uint32_t bar_full = smem_u32(bars), bar_empty = bar_full + 8 * NSTG, bar_acc = bar_full + 16 * NSTG;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int tn = blockIdx.x, tm = blockIdx.y;
  const int rows = npts * R;

  if (threadIdx.x == 0) {
    for (int s = 0; s < NSTG; ++s) {
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

  if (warp == 0) {
    if (lane == 0) {
      for (int kc = 0; kc < nkc; ++kc) {
        const int s = kc % NSTG;
        if (kc >= NSTG && !mbar_wait(bar_empty + 8 * s, ((kc / NSTG) - 1) & 1, err, 31)) break;
        const uint32_t st = sbase + s * STG;
        mbar_expect_tx(bar_full + 8 * s, STG);
#pragma unroll 1
        for (int q = 0; q < S; ++q) {
          tma_load_3d(st + q * A_SL, &mapA, bar_full + 8 * s, kc * KC, tm * RB_M, ch * S + q);
          tma_load_3d(st + S * A_SL + q * B_SL, &mapB, bar_full + 8 * s, kc * KC, tn * RB_N, ch * S + q);
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      bool ok = true;
      for (int kc = 0; kc < nkc && ok; ++kc) {
        const int s = kc % NSTG;
        if (!(ok = mbar_wait(bar_full + 8 * s, (kc / NSTG) & 1, err, 32))) break;
        asm volatile("tcgen05.fence::after_thread_sync;");
        const uint32_t st = sbase + s * STG;
        // group g = p + q (p, q = 1..S, g <= S + 1) into accumulator g - 2
#pragma unroll 1
        for (int gi = 0; gi < NG; ++gi) {
          const uint32_t dacc = tmem + (uint32_t)(gi * RB_N);
#pragma unroll 1
          for (int p = 1; p <= gi + 1; ++p) {
            const int q = gi + 2 - p;
#pragma unroll
            for (int k2 = 0; k2 < 2; ++k2) {
              const uint64_t da = desc_sw64(st + (p - 1) * A_SL + 32 * k2);
              const uint64_t db = desc_sw64(st + S * A_SL + (q - 1) * B_SL + 32 * k2);
              mma_i8(dacc, da, db, (kc > 0 || p > 1 || k2 > 0) ? 1u : 0u);
            }
          }
        }
        mma_commit(bar_empty + 8 * s);
      }
      if (ok) mma_commit(bar_acc);
    }
  } else if (warp >= 4) {
    const int e4 = warp - 4, quad = warp & 3, half = e4 >> 2;
    const int row = tm * RB_M + quad * 32 + lane;
    bool ok = mbar_wait(bar_acc, 0, err, 33);
    if (__all_sync(0xffffffffu, ok)) {
      asm volatile("tcgen05.fence::after_thread_sync;");
      double are[16], aim[16];
#pragma unroll
      for (int j = 0; j < 16; ++j) are[j] = aim[j] = 0.0;
      const uint32_t tl = tmem + ((uint32_t)(quad * 32) << 16) + (uint32_t)(half * 16);
      // groups from the smallest weight up: sum_g 2^(-7 g) G_g
#pragma unroll 1
      for (int gi = NG - 1; gi >= 0; --gi) {
        int gre[16], gim[16];
        tmem_ld16i(tl + gi * RB_N, gre);
        tmem_ld16i(tl + gi * RB_N + RB_N / 2, gim);
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        const double w = ldexp(1.0, -7 * (gi + 2));
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          are[j] = fma((double)gre[j], w, are[j]);
          aim[j] = fma((double)gim[j], w, aim[j]);
        }
      }
      if (row < rows) {
        const int p = row / R, i1 = row % R;
        const size_t m = (size_t)(2 * p + ch), per = (size_t)R * N;
        const int ea = eA[(size_t)ch * rows_cap + row];
        double rmax = 0.0;
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int c = tn * (RB_N / 2) + half * 16 + j;
          if (c >= N) continue;
          const int sc = ea + eB[(size_t)ch * N + c] + 2;
          const size_t o = m * per + (size_t)i1 * N + c;
          const z64 b = Bpt ? Bpt[o] : opg[i1 + (size_t)c * R];
          const z64 x = X[o];
          z64 r = make_double2(b.x - x.x + ldexp(are[j], sc), b.y - x.y + ldexp(aim[j], sc));
          if (extra) r = cadd(r, extra[(size_t)p * per + (size_t)i1 * N + c]);   // V(q) term (density)
          V[o] = to32(r);
          rmax = fmax(rmax, fabs(r.x) + fabs(r.y));
        }
        if (rnorm && rmax > 0.0) atomicMax(rnorm + m, (unsigned long long)__double_as_longlong(rmax));
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 1) {
    asm volatile("tcgen05.fence::after_thread_sync;");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS));
  }
}

// int8 slices [planes][rows][K2p], box 64 B x box_rows, 64 B swizzle
bool make_map_i8(CUtensorMap *map, void *base, uint64_t K2p, uint64_t rows, uint64_t planes, uint32_t box_rows) {
  encode_fn_t enc = tmap_encoder();
  if (!enc) return false;
  cuuint64_t dims[3] = {K2p, rows, planes};
  cuuint64_t strides[2] = {K2p, K2p * rows};
  cuuint32_t box[3] = {(cuuint32_t)KC, box_rows, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  return enc(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
             CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

struct RiCtx {
  int N, R, cap;
  int K2p, N2p;
  size_t rows_cap;
  signed char *As = nullptr, *Bs = nullptr;
  int *eA = nullptr, *eB = nullptr, *err = nullptr;
  CUtensorMap mapA, mapB;
  const void *f_key[2] = {nullptr, nullptr};   // F~ of the current slices, per channel
  long long f_gen[2] = {-1, -1};
};

}  // namespace

// Slices and maps for batches of up to `cap` points (N, R of the handle).
cudaError_t ri8_setup(void **ctx_out, int N, int R, int cap) {
  *ctx_out = nullptr;
  RiCtx *c = new RiCtx();
  c->N = N;
  c->R = R;
  c->cap = cap;
  c->K2p = (2 * N + KC - 1) / KC * KC;
  c->N2p = (2 * N + RB_N - 1) / RB_N * RB_N;
  c->rows_cap = (size_t)cap * R;
  cudaError_t e = cudaMalloc(&c->As, (size_t)2 * S * c->rows_cap * c->K2p);
  if (e == cudaSuccess) e = cudaMalloc(&c->Bs, (size_t)2 * S * c->N2p * c->K2p);
  if (e == cudaSuccess) e = cudaMalloc(&c->eA, sizeof(int) * 2 * c->rows_cap);
  if (e == cudaSuccess) e = cudaMalloc(&c->eB, sizeof(int) * 2 * N);
  if (e == cudaSuccess) e = cudaMalloc(&c->err, sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(c->err, 0, sizeof(int));
  if (e == cudaSuccess && (!make_map_i8(&c->mapA, c->As, c->K2p, c->rows_cap, 2 * S, RB_M) ||
                           !make_map_i8(&c->mapB, c->Bs, c->K2p, c->N2p, 2 * S, RB_N)))
    e = cudaErrorInvalidValue;
  if (e == cudaSuccess) e = smem_limit(k_resid_i8, RI_SMEM);
  if (e != cudaSuccess) {
    cudaFree(c->As); cudaFree(c->Bs); cudaFree(c->eA); cudaFree(c->eB); cudaFree(c->err);
    delete c;
    return e;
  }
  *ctx_out = c;
  return cudaSuccess;
}

void ri8_free(void *ctxp) {
  RiCtx *c = (RiCtx *)ctxp;
  if (!c) return;
  cudaFree(c->As); cudaFree(c->Bs); cudaFree(c->eA); cudaFree(c->eB); cudaFree(c->err);
  delete c;
}

int ri8_error(void *ctxp) {
  RiCtx *c = (RiCtx *)ctxp;
  int v = 0;
  if (!c || cudaMemcpy(&v, c->err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
  return v;
}

// r = B - X + XD F~ for both channels of a batch of npts points (npts <= cap): the
// slices of F~ are cut again only when (Frow, fgen) changed
cudaError_t ri8_residual(void *ctxp, const DevCtx &dc, int npts, const z64 *XD, const z64 *X,
                         const z64 *Frow_d, const z64 *Frow_m, long long fgen, const z64 *opg_d,
                         const z64 *opg_m, z32 *V, const z64 *extra_d, unsigned long long *rnorm, const z64 *Bpt,
                         cudaStream_t st) {
  RiCtx *c = (RiCtx *)ctxp;
  if (!c || npts > c->cap || dc.N != c->N || dc.R != c->R) return cudaErrorInvalidValue;
  const int rows = npts * c->R;
  const int nkc = c->K2p / KC;
  for (int ch = 0; ch < 2; ++ch) {
    const z64 *F = ch ? Frow_m : Frow_d;
    if (c->f_key[ch] != F || c->f_gen[ch] != fgen) {
      k_slice_cols<<<cdiv_u((size_t)c->N2p * 32, 256), 256, 0, st>>>(c->N, ch, F, c->Bs, c->eB, c->K2p, c->N2p);
      cudaError_t e = ADGA_LAUNCH_CHECK();
      if (e != cudaSuccess) return e;
      c->f_key[ch] = F;
      c->f_gen[ch] = fgen;
    }
    k_slice_rows<<<cdiv_u((size_t)rows * 32, 256), 256, 0, st>>>(c->N, c->R, npts, ch, XD, c->As, c->eA, c->K2p,
                                                                  c->rows_cap);
    cudaError_t e = ADGA_LAUNCH_CHECK();
    if (e != cudaSuccess) return e;
    dim3 grid(c->N2p / RB_N, cdiv_u(rows, RB_M));
    k_resid_i8<<<grid, RI_THREADS, RI_SMEM, st>>>(c->mapA, c->mapB, c->N, c->R, npts, ch, nkc, c->eA, c->eB,
                                                  c->rows_cap, X, ch ? opg_m : opg_d, V, ch ? nullptr : extra_d,
                                                  rnorm, Bpt, c->err);
    if ((e = ADGA_LAUNCH_CHECK()) != cudaSuccess) return e;
  }
  return cudaSuccess;
}
