// Streaming blocked triangular solves for the batched LU (few right-hand
// sides), and the row permutation of a factorization.
//
// The solve L Y = P B (unit-lower, forward) or U X = Y (upper, backward) for
// R <= 25 right-hand sides reads the whole triangle once and does R complex
// FMAs per element read, so it is bound by HBM bandwidth.  One CTA solves
// one matrix; the triangle's NB-column panels reach shared memory through a
// STAGES-deep cp.async ring (256 rows x 16 columns per stage: 32 KB FP32,
// 64 KB FP64), so that the next tiles are in flight while the current one is
// applied:
//
//   per block step (NB = 64 columns J..J+jb):
//     D item   the inverted diagonal block (from k_triinv) -> stage;
//              Y = D^-1 B[J..J+jb] (one thread per (row, rhs)), written back
//              to B and kept in shared memory;
//     U items  for each 256-row chunk of the rows still to solve and each
//              16-column slice of the panel: acc += L[rows, cols] Y[cols];
//              after the last slice B[rows] -= acc.
//
// The right-hand sides stay in global memory (the forward solve gathers P B
// into a work copy first): a CTA's 10-80 KB of them stay in L2, and leaving
// shared memory to the ring keeps two FP32 CTAs per SM.  Thread (il, g) of
// a U item owns two rows of the chunk and RG right-hand sides g*RG..:
// FP32 takes the adjacent rows 2 il, 2 il + 1 with one 16-byte load and
// keeps their real and imaginary parts as lane pairs of packed two-lane
// FMAs (__ffma2_rn) against Y stored as (re, re, im, im); FP64 takes rows
// il and il + 128.
//
// The reference inverts with zgetrf + zgetri (src/lapack_module.f90:40-70);
// the solves here use the same factorization as LAPACK's zgetrs does: B is
// permuted by the row interchanges ipiv[0], ipiv[1], ... applied in order
// (zlaswp), as one permutation precomputed per factorization by k_build_perm.
#include "lu.cuh"

namespace {

constexpr int TS_NB = 64;               // block width the solve is written for
constexpr int TS_CH = 256;              // rows per U item
constexpr int TS_KS = 16;               // panel columns per U item
// bytes per ring stage: one U item, or one NB x NB diagonal block
template <typename T> __host__ __device__ constexpr int ts_stage() { return TS_CH * TS_KS * (int)sizeof(T); }
static_assert(TS_NB * TS_NB <= TS_CH * TS_KS, "a diagonal block must fit one stage");

// Y as the U items read it: FP32 (re, re, im, im) lane pairs, FP64 plain
template <typename T> struct TsY;
template <> struct TsY<z32> { typedef float4 type; };
template <> struct TsY<z64> { typedef double2 type; };

__device__ __forceinline__ void ts_cp16(void *smem, const void *gmem) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void ts_commit() { asm volatile("cp.async.commit_group;"); }
template <int N> __device__ __forceinline__ void ts_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// position in the item sequence: step s, chunk c (-1 = the D item), slice kh
struct TsIt {
  int s, c, kh;
};

struct TsGeo {
  int blk, J, jb, rb, re, nch, nkh;
};

template <bool UPPER, int KS>
__device__ __forceinline__ TsGeo ts_geo(int s, int N, int nsteps) {
  TsGeo g;
  g.blk = UPPER ? nsteps - 1 - s : s;
  g.J = g.blk * TS_NB;
  g.jb = min(TS_NB, N - g.J);
  g.rb = UPPER ? 0 : g.J + g.jb;
  g.re = UPPER ? g.J : N;
  g.nch = (g.re - g.rb + TS_CH - 1) / TS_CH;
  g.nkh = (g.jb + KS - 1) / KS;
  return g;
}

template <bool UPPER, int KS>
__device__ __forceinline__ void ts_next(TsIt &it, int N, int nsteps) {
  const TsGeo g = ts_geo<UPPER, KS>(it.s, N, nsteps);
  if (it.c < 0) {
    it.c = 0;
    it.kh = 0;
  } else if (++it.kh >= g.nkh) {
    it.kh = 0;
    ++it.c;
  }
  if (it.c >= g.nch) {
    ++it.s;
    it.c = -1;
    it.kh = 0;
  }
}

__device__ __forceinline__ float4 ts_pack(float2 y) { return make_float4(y.x, y.x, y.y, y.y); }
__device__ __forceinline__ double2 ts_pack(double2 y) { return y; }

}  // namespace

// perm[b][i] = source row of row i of P B (ipiv 0-based, applied in order)
__global__ void k_build_perm(const int *__restrict__ ipiv_all, int N, int *__restrict__ perm_all) {
  extern __shared__ int sh_perm[];
  int *ip = sh_perm, *pm = sh_perm + N;
  const int b = blockIdx.x, t = threadIdx.x;
  for (int i = t; i < N; i += blockDim.x) {
    ip[i] = ipiv_all[(size_t)b * N + i];
    pm[i] = i;
  }
  __syncthreads();
  if (t == 0)
    for (int i = 0; i < N; ++i) {
      const int p = ip[i];
      if (p != i && p >= 0 && p < N) {
        const int x = pm[i];
        pm[i] = pm[p];
        pm[p] = x;
      }
    }
  __syncthreads();
  for (int i = t; i < N; i += blockDim.x) perm_all[(size_t)b * N + i] = pm[i];
}

template <typename T, bool UPPER, int RG, int NG, int STAGES>
__global__ void __launch_bounds__(128 * NG, sizeof(T) == 8 && NG <= 3 ? 2 : 1)
k_trsv_stream(const T *__restrict__ M, size_t strideM, int N, int nsteps, const T *__restrict__ Dinv,
              T *C, size_t strideC, int ldc, int R, const int *__restrict__ perm_all, T *work) {
  constexpr int NT = 128 * NG;
  constexpr int KS = TS_KS;
  constexpr int TS_STAGE = ts_stage<T>();
  constexpr bool F32 = sizeof(T) == 8;
  typedef typename TsY<T>::type YT;
  extern __shared__ __align__(16) unsigned char smraw[];
  constexpr int RP = RG * NG;   // right-hand sides padded to the thread groups
  YT *Ys = reinterpret_cast<YT *>(smraw + (size_t)STAGES * TS_STAGE);   // [NB][RP]
  T *Cbs = reinterpret_cast<T *>(Ys + TS_NB * RP);                        // [R][NB]
  const int b = blockIdx.x, t = threadIdx.x;
  const T *A = M + (size_t)b * strideM;
  T *X;
  int ldx;
  if (!UPPER) {
    // P B into the work copy: row i of P B is row perm[i] of B
    X = work + (size_t)b * N * R;
    ldx = N;
    const int *perm = perm_all + (size_t)b * N;
    const T *Cb = C + (size_t)b * strideC;
    // eight loads in flight per thread before their stores (X and C could
    // alias as far as the compiler knows)
    for (int e0 = 0; e0 < N * R; e0 += 8 * NT) {
      T v[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int e = e0 + u * NT + t;
        if (e < N * R) v[u] = Cb[(size_t)perm[e % N] + (size_t)(e / N) * ldc];
      }
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int e = e0 + u * NT + t;
        if (e < N * R) X[e] = v[u];
      }
    }
  } else {
    X = C + (size_t)b * strideC;
    ldx = ldc;
  }

  auto issue = [&](const TsIt &it, int slot) {
    if (it.s < nsteps) {
      const TsGeo g = ts_geo<UPPER, KS>(it.s, N, nsteps);
      unsigned char *dst = smraw + (size_t)slot * TS_STAGE;
      if (it.c < 0) {
        const unsigned char *src =
            reinterpret_cast<const unsigned char *>(Dinv + ((size_t)b * nsteps + g.blk) * TS_NB * TS_NB);
        constexpr int pieces = TS_NB * TS_NB * (int)sizeof(T) / 16;
        for (int e = t; e < pieces; e += NT) ts_cp16(dst + 16 * e, src + 16 * e);
      } else {
        const int r0 = g.rb + it.c * TS_CH, nr = min(TS_CH, g.re - r0);
        const int k0 = g.J + it.kh * KS, kc = min(KS, g.jb - it.kh * KS);
        // a column holds PPC 16-byte pieces (a power of two); the chunk's nr rows fill ppc of them
        constexpr int PPC = TS_CH * (int)sizeof(T) / 16;
        const int ppc = nr * (int)sizeof(T) / 16;
        const unsigned char *src0 = reinterpret_cast<const unsigned char *>(A + (size_t)k0 * N + r0);
        constexpr int TRIPS = (KS * PPC + NT - 1) / NT;
#pragma unroll
        for (int u = 0; u < TRIPS; ++u) {
          const int e = t + u * NT, kk = e / PPC, p = e % PPC;
          if (kk < kc && p < ppc)
            ts_cp16(dst + (size_t)kk * TS_CH * sizeof(T) + 16 * p, src0 + ((size_t)kk * N * sizeof(T) + 16 * p));
        }
      }
    }
    ts_commit();
  };

  // padded right-hand sides r >= R read zeros (their results are never stored)
  for (int e = t; e < TS_NB * (RP - R); e += NT) Ys[(e / (RP - R)) * RP + R + e % (RP - R)] = YT{};
  TsIt pit{0, -1, 0}, cit{0, -1, 0};
#pragma unroll
  for (int i = 0; i < STAGES - 1; ++i) {
    issue(pit, i);
    ts_next<UPPER, KS>(pit, N, nsteps);
  }
  const int il = t & 127, gq = t >> 7;
  T acc0[RG], acc1[RG];
  for (int gidx = 0; cit.s < nsteps; ++gidx) {
    ts_wait<STAGES - 2>();
    __syncthreads();
    issue(pit, (gidx + STAGES - 1) % STAGES);
    ts_next<UPPER, KS>(pit, N, nsteps);
    const T *S = reinterpret_cast<const T *>(smraw + (size_t)(gidx % STAGES) * TS_STAGE);
    const TsGeo g = ts_geo<UPPER, KS>(cit.s, N, nsteps);
    if (cit.c < 0) {
      // ---- diagonal block: Y = D^-1 B[J..J+jb]
      for (int e = t; e < g.jb * R; e += NT) {
        const int k = e % g.jb, r = e / g.jb;
        Cbs[r * TS_NB + k] = X[(size_t)(g.J + k) + (size_t)r * ldx];
      }
      __syncthreads();
      for (int e = t; e < g.jb * R; e += NT) {
        const int i = e % g.jb, r = e / g.jb;
        const int kb = UPPER ? i : 0, ke = UPPER ? g.jb : i + 1;
        T v0 = czero<T>(), v1 = czero<T>(), v2 = czero<T>(), v3 = czero<T>();
        const T *cb = Cbs + r * TS_NB;
        int k = kb;
        for (; k + 3 < ke; k += 4) {
          cfma(v0, S[i + k * TS_NB], cb[k]);
          cfma(v1, S[i + (k + 1) * TS_NB], cb[k + 1]);
          cfma(v2, S[i + (k + 2) * TS_NB], cb[k + 2]);
          cfma(v3, S[i + (k + 3) * TS_NB], cb[k + 3]);
        }
        for (; k < ke; ++k) cfma(v0, S[i + k * TS_NB], cb[k]);
        const T y = cadd(cadd(v0, v1), cadd(v2, v3));
        X[(size_t)(g.J + i) + (size_t)r * ldx] = y;
        Ys[i * RP + r] = ts_pack(y);
      }
    } else {
      // ---- update slice: acc += L[rows, cols] Y[cols]; B[rows] -= acc after the last slice
      const int r0 = g.rb + cit.c * TS_CH, nr = min(TS_CH, g.re - r0);
      const int kc = min(KS, g.jb - cit.kh * KS);
      const bool last = cit.kh == g.nkh - 1;
      const YT *yb = Ys + cit.kh * KS * RP + gq * RG;
      // FP32: rows (2 il, 2 il + 1) as lane pairs; FP64: rows il and il + 128
      const int ra = F32 ? 2 * il : il, rbb = F32 ? 2 * il + 1 : il + 128;
      if (cit.kh == 0) {
#pragma unroll
        for (int j = 0; j < RG; ++j) acc0[j] = acc1[j] = czero<T>();
      }
      // the right-hand sides of the last slice are loaded before its k loop
      T b0[RG], b1[RG];
      if (last) {
#pragma unroll
        for (int j = 0; j < RG; ++j) {
          const int r = gq * RG + j;
          b0[j] = (r < R && ra < nr) ? X[(size_t)(r0 + ra) + (size_t)r * ldx] : czero<T>();
          b1[j] = (r < R && rbb < nr) ? X[(size_t)(r0 + rbb) + (size_t)r * ldx] : czero<T>();
        }
      }
      if constexpr (F32) {
        // acc0[j] = real parts of the two rows, acc1[j] = imaginary parts
        const float4 *S4 = reinterpret_cast<const float4 *>(S);
#pragma unroll 4
        for (int kk = 0; kk < kc; ++kk) {
          const float4 a = S4[kk * (TS_CH / 2) + il];
          const float2 ar = make_float2(a.x, a.z), ai = make_float2(a.y, a.w);
#pragma unroll
          for (int j = 0; j < RG; ++j) {
            const float4 q = yb[kk * RP + j];
            const float2 yr = make_float2(q.x, q.y), yi = make_float2(q.z, q.w);
            acc0[j] = __ffma2_rn(ar, yr, acc0[j]);
            acc0[j] = __ffma2_rn(ai, make_float2(-q.z, -q.w), acc0[j]);
            acc1[j] = __ffma2_rn(ar, yi, acc1[j]);
            acc1[j] = __ffma2_rn(ai, yr, acc1[j]);
          }
        }
        if (last) {
#pragma unroll
          for (int j = 0; j < RG; ++j) {
            const int r = gq * RG + j;
            if (r < R) {
              if (ra < nr)
                X[(size_t)(r0 + ra) + (size_t)r * ldx] = csub(b0[j], make_float2(acc0[j].x, acc1[j].x));
              if (rbb < nr)
                X[(size_t)(r0 + rbb) + (size_t)r * ldx] = csub(b1[j], make_float2(acc0[j].y, acc1[j].y));
            }
          }
        }
      } else {
#pragma unroll 4
        for (int kk = 0; kk < kc; ++kk) {
          const T a0 = S[kk * TS_CH + il], a1 = S[kk * TS_CH + il + 128];
#pragma unroll
          for (int j = 0; j < RG; ++j) {
            const YT y = yb[kk * RP + j];
            cfma(acc0[j], a0, y);
            cfma(acc1[j], a1, y);
          }
        }
        if (last) {
#pragma unroll
          for (int j = 0; j < RG; ++j) {
            const int r = gq * RG + j;
            if (r < R) {
              if (ra < nr) X[(size_t)(r0 + ra) + (size_t)r * ldx] = csub(b0[j], acc0[j]);
              if (rbb < nr) X[(size_t)(r0 + rbb) + (size_t)r * ldx] = csub(b1[j], acc1[j]);
            }
          }
        }
      }
    }
    ts_next<UPPER, KS>(cit, N, nsteps);
  }
  ts_wait<0>();
  if (!UPPER) {
    __syncthreads();
    T *Cb = C + (size_t)b * strideC;
    for (int e0 = 0; e0 < N * R; e0 += 8 * NT) {
      T v[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int e = e0 + u * NT + t;
        if (e < N * R) v[u] = X[e];
      }
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int e = e0 + u * NT + t;
        if (e < N * R) Cb[(size_t)(e % N) + (size_t)(e / N) * ldc] = v[u];
      }
    }
  }
}

cudaError_t lu_build_perm(const LUBatch &lb, int *perm, cudaStream_t st) {
  if (!perm || lb.N > 8192) return cudaErrorInvalidValue;
  k_build_perm<<<lb.batch, 128, sizeof(int) * 2 * lb.N, st>>>(lb.ipiv, lb.N, perm);
  return ADGA_LAUNCH_CHECK();
}

// Shared memory of the streaming solve: the ring, Y and the staged block of B.
template <typename T> static size_t ts_smem(int R, int RP, int stages) {
  return (size_t)stages * ts_stage<T>() + sizeof(typename TsY<T>::type) * TS_NB * RP + sizeof(T) * TS_NB * R;
}

template <typename T>
bool trsv_stream_supported(const LUBatch &lb, size_t strideC, int R, bool upper, const int *perm,
                           const T *work) {
  if (lb.NB != TS_NB || R < 1 || R > 25) return false;
  if (!upper && (!perm || !work)) return false;
  // 16-byte cp.async pieces: every panel column segment must start and end on 16 bytes
  if (sizeof(T) == 8 && ((lb.N & 1) || (lb.strideM & 1))) return false;
  (void)strideC;
  const int RP = R == 1 ? 1 : R <= 4 ? 4 : R <= 9 ? 9 : R <= 16 ? 16 : 25;
  return ts_smem<T>(R, RP, R > 16 ? 2 : 3) <= 227 * 1024;
}

template <typename T>
cudaError_t launch_trsv_stream(const T *M, const LUBatch &lb, T *C, size_t strideC, int ldc, int R,
                               bool upper, const int *perm, T *work, cudaStream_t st) {
  const int np = lb.nsteps();
  const T *D = (const T *)(upper ? lb.Uinv : lb.Linv);
#define TSV(UP, RGV, NGV, STG)                                                                     \
  do {                                                                                             \
    const size_t sm = ts_smem<T>(R, RGV * NGV, STG);                                                          \
    smem_limit(k_trsv_stream<T, UP, RGV, NGV, STG>, 227 * 1024);                                   \
    k_trsv_stream<T, UP, RGV, NGV, STG><<<lb.batch, 128 * NGV, sm, st>>>(                          \
        M, lb.strideM, lb.N, np, D, C, strideC, ldc, R, perm, work);                               \
  } while (0)
#define TSV_R(UP)                                                                                  \
  do {                                                                                             \
    if (R == 1) TSV(UP, 1, 1, 3);                                                                  \
    else if (R <= 4) TSV(UP, 2, 2, 3);                                                             \
    else if (R <= 9) TSV(UP, 3, 3, 3);                                                             \
    else if (R <= 16) TSV(UP, 4, 4, 3);                                                            \
    else TSV(UP, 5, 5, 2);                                                                         \
  } while (0)
  if (upper) TSV_R(true);
  else TSV_R(false);
#undef TSV_R
#undef TSV
  return ADGA_LAUNCH_CHECK();
}

template bool trsv_stream_supported<z32>(const LUBatch &, size_t, int, bool, const int *, const z32 *);
template bool trsv_stream_supported<z64>(const LUBatch &, size_t, int, bool, const int *, const z64 *);
template cudaError_t launch_trsv_stream<z32>(const z32 *, const LUBatch &, z32 *, size_t, int, int, bool,
                                             const int *, z32 *, cudaStream_t);
template cudaError_t launch_trsv_stream<z64>(const z64 *, const LUBatch &, z64 *, size_t, int, int, bool,
                                             const int *, z64 *, cudaStream_t);
