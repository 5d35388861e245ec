// Batched blocked right-looking LU with partial pivoting (complex FP64 or
// FP32) and blocked triangular solves; see lu.cuh for the layout.
//
// Per step J (panel width NB):
//   k_panel      one CTA per matrix factors rows J..N of the NB panel columns
//                in 8-column sub-panels held in registers (pivot search,
//                row swap and rank-1 updates never leave the SM), with
//                right-looking rank-8 updates of the rest of the panel;
//   k_triinv     inverts the unit-lower and upper NB x NB diagonal blocks;
//   k_swap_trsm  applies the panel's row interchanges to the other columns
//                and forms U12 = L11^-1 A12 as a small GEMM;
//   trailing     A22 -= L21 U12 (CUDA-core GEMM below, or the tensor-core
//                BF16x3 kernel of the mixed path).
// Pivot choice follows izamax: the largest |re|+|im|, the lowest row on ties.
#include "lu.cuh"
#include <climits>

#define SWD 8          // sub-panel width
#define MAXNB 128      // largest outer panel width

// ---------------------------------------------------------------------------
template <int RPT> struct PanelThreads { static constexpr int v = RPT == 1 ? 1024 : RPT == 2 ? 640 : 512; };

template <typename T> struct PanelShared {
  typename cx<T>::real red_v[32];
  int red_i[32];
  int s_p;
  int s_info;
  int s_piv[SWD];
  int mdst[2 * SWD], msrc[2 * SWD];
  int mcnt;
  T bufP[SWD], bufC[SWD];
  T Lss[SWD * SWD];
  T Us[SWD * MAXNB];
};

// One column CC of the register-resident sub-panel: pivot search, row swap,
// scaling and rank-1 update.  CC is a compile-time constant so that every
// index into the register array a[][] is static.
template <typename T, int RPT, int CC>
__device__ __forceinline__ void panel_column(T (&a)[RPT][SWD], PanelShared<T> &S, int J, int N,
                                             int c0, int sw, int t, int nt) {
  typedef typename cx<T>::real R;
  if (CC >= sw) return;
  const int lane = t & 31, warp = t >> 5, nw = nt >> 5;
  const int col = c0 + CC;
  R best = R(-1);
  int bidx = INT_MAX;
#pragma unroll
  for (int q = 0; q < RPT; ++q) {
    const int r = J + t + q * nt;
    if (r >= col && r < N) {
      R v = cabs1(a[q][CC]);
      if (v > best) { best = v; bidx = r; }
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    R ov = __shfl_xor_sync(0xffffffffu, best, o);
    int oi = __shfl_xor_sync(0xffffffffu, bidx, o);
    if (ov > best || (ov == best && oi < bidx)) { best = ov; bidx = oi; }
  }
  if (lane == 0) { S.red_v[warp] = best; S.red_i[warp] = bidx; }
  __syncthreads();
  if (warp == 0) {
    best = lane < nw ? S.red_v[lane] : R(-1);
    bidx = lane < nw ? S.red_i[lane] : INT_MAX;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      R ov = __shfl_xor_sync(0xffffffffu, best, o);
      int oi = __shfl_xor_sync(0xffffffffu, bidx, o);
      if (ov > best || (ov == best && oi < bidx)) { best = ov; bidx = oi; }
    }
    if (lane == 0) S.s_p = (bidx == INT_MAX || bidx < col || bidx >= N) ? col : bidx;
  }
  __syncthreads();
  const int p = S.s_p;
  const int oc = col - J, op = p - J;
  const bool own_c = (oc % nt) == t, own_p = (op % nt) == t;
  const int qc = oc / nt, qp = op / nt;
#pragma unroll
  for (int q = 0; q < RPT; ++q) {
    if (own_p && q == qp)
#pragma unroll
      for (int c2 = 0; c2 < SWD; ++c2) S.bufP[c2] = a[q][c2];
    if (own_c && q == qc)
#pragma unroll
      for (int c2 = 0; c2 < SWD; ++c2) S.bufC[c2] = a[q][c2];
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < RPT; ++q) {
    if (own_c && q == qc)
#pragma unroll
      for (int c2 = 0; c2 < SWD; ++c2) a[q][c2] = S.bufP[c2];
    if (own_p && p != col && q == qp)
#pragma unroll
      for (int c2 = 0; c2 < SWD; ++c2) a[q][c2] = S.bufC[c2];
  }
  const T piv = S.bufP[CC];
  const bool zero = (piv.x == R(0) && piv.y == R(0));
  if (zero && t == 0 && S.s_info == 0) S.s_info = col + 1;
  const T rcp = zero ? czero<T>() : crcp(piv);
  T prow[SWD];
#pragma unroll
  for (int c2 = CC + 1; c2 < SWD; ++c2) prow[c2] = S.bufP[c2];
#pragma unroll
  for (int q = 0; q < RPT; ++q) {
    const int r = J + t + q * nt;
    if (r > col && r < N) {
      const T l = zero ? a[q][CC] : cmul(a[q][CC], rcp);
      a[q][CC] = l;
#pragma unroll
      for (int c2 = CC + 1; c2 < SWD; ++c2)
        if (c2 < sw) cfms(a[q][c2], l, prow[c2]);
    }
  }
  if (t == 0) S.s_piv[CC] = p;
}

template <typename T, int RPT>
__global__ void __launch_bounds__(PanelThreads<RPT>::v, 1)
k_panel(T *M, size_t strideM, int N, int J, int jb, int *ipiv_all, int *info_all) {
  const int b = blockIdx.x;
  T *A = M + (size_t)b * strideM;
  int *ipiv = ipiv_all + (size_t)b * N;
  const int nt = blockDim.x, t = threadIdx.x;
  __shared__ PanelShared<T> S;
  extern __shared__ __align__(16) unsigned char panel_dyn[];
  T *Gs = reinterpret_cast<T *>(panel_dyn);        // [MAXNB][2*SWD] interchange buffer
  if (t == 0) S.s_info = info_all[b];
  T a[RPT][SWD];

  for (int s = 0; s < jb; s += SWD) {
    const int sw = min(SWD, jb - s), c0 = J + s;
#pragma unroll
    for (int q = 0; q < RPT; ++q) {
      const int r = J + t + q * nt;
#pragma unroll
      for (int cc = 0; cc < SWD; ++cc)
        a[q][cc] = (r >= c0 && r < N && cc < sw) ? A[r + (size_t)(c0 + cc) * N] : czero<T>();
    }
    panel_column<T, RPT, 0>(a, S, J, N, c0, sw, t, nt);
    panel_column<T, RPT, 1>(a, S, J, N, c0, sw, t, nt);
    panel_column<T, RPT, 2>(a, S, J, N, c0, sw, t, nt);
    panel_column<T, RPT, 3>(a, S, J, N, c0, sw, t, nt);
    panel_column<T, RPT, 4>(a, S, J, N, c0, sw, t, nt);
    panel_column<T, RPT, 5>(a, S, J, N, c0, sw, t, nt);
    panel_column<T, RPT, 6>(a, S, J, N, c0, sw, t, nt);
    panel_column<T, RPT, 7>(a, S, J, N, c0, sw, t, nt);
    // ---- write the sub-panel back; keep its L block for the TRSM below
#pragma unroll
    for (int q = 0; q < RPT; ++q) {
      const int r = J + t + q * nt;
      if (r >= c0 && r < N) {
#pragma unroll
        for (int cc = 0; cc < SWD; ++cc)
          if (cc < sw) A[r + (size_t)(c0 + cc) * N] = a[q][cc];
        const int i = r - c0;
        if (i < sw)
#pragma unroll
          for (int cc = 0; cc < SWD; ++cc) S.Lss[i + cc * SWD] = a[q][cc];
      }
    }
    if (t == 0) {
      // compose the sub-panel's interchanges into a (dst <- src) row map
      int keys[2 * SWD], cont[2 * SWD], nk = sw;
      for (int i = 0; i < sw; ++i) { keys[i] = c0 + i; cont[i] = c0 + i; }
      for (int i = 0; i < sw; ++i) {
        const int p = S.s_piv[i];
        if (p == c0 + i) continue;
        int k = -1;
        if (p < c0 + sw) k = p - c0;
        else {
          for (int q = sw; q < nk; ++q)
            if (keys[q] == p) { k = q; break; }
          if (k < 0) { k = nk++; keys[k] = p; cont[k] = p; }
        }
        const int x = cont[i]; cont[i] = cont[k]; cont[k] = x;
      }
      int cnt = 0;
      for (int k = 0; k < nk; ++k)
        if (cont[k] != keys[k]) { S.mdst[cnt] = keys[k]; S.msrc[cnt] = cont[k]; ++cnt; }
      S.mcnt = cnt;
    }
    __syncthreads();
    if (t < sw) ipiv[c0 + t] = S.s_piv[t];
    // ---- apply the sub-panel's interchanges to the other panel columns:
    //      every (row, column) load into shared memory, a barrier, every store
    const int nother = jb - sw, mc = S.mcnt;
    for (int e = t; e < nother * mc; e += nt) {
      const int u = e / mc, k = e % mc;
      const int col = (u < s) ? J + u : c0 + sw + (u - s);
      Gs[u * 2 * SWD + k] = A[(size_t)S.msrc[k] + (size_t)col * N];
    }
    __syncthreads();
    for (int e = t; e < nother * mc; e += nt) {
      const int u = e / mc, k = e % mc;
      const int col = (u < s) ? J + u : c0 + sw + (u - s);
      A[(size_t)S.mdst[k] + (size_t)col * N] = Gs[u * 2 * SWD + k];
    }
    __syncthreads();
    // ---- U rows of the right panel columns: unit-lower solve with Lss
    const int nright = jb - s - sw;
    for (int u = t; u < nright; u += nt) {
      const int col = c0 + sw + u;
      T *Ac = A + (size_t)col * N;
      T x[SWD];
#pragma unroll
      for (int i = 0; i < SWD; ++i) x[i] = (i < sw) ? Ac[c0 + i] : czero<T>();
#pragma unroll
      for (int i = 1; i < SWD; ++i)
#pragma unroll
        for (int k = 0; k < i; ++k) cfms(x[i], S.Lss[i + k * SWD], x[k]);
#pragma unroll
      for (int i = 0; i < SWD; ++i)
        if (i < sw) { Ac[c0 + i] = x[i]; S.Us[i * MAXNB + u] = x[i]; }
    }
    __syncthreads();
    // ---- rank-sw update of the rows below, right panel columns, in chunks of
    //      CW columns whose loads are all issued before their stores (CW
    //      keeps the chunk beside a[][] inside the register budget)
    if (nright > 0) {
#pragma unroll
      for (int q = 0; q < RPT; ++q) {
        const int r = J + t + q * nt;
        if (r >= c0 + sw && r < N) {
          T *arow = A + r + (size_t)(c0 + sw) * N;
          constexpr int CW = sizeof(T) == 8 ? 4 : 2;
          for (int u0 = 0; u0 < nright; u0 += CW) {
            T v[CW];
#pragma unroll
            for (int j = 0; j < CW; ++j)
              if (u0 + j < nright) v[j] = arow[(size_t)(u0 + j) * N];
#pragma unroll
            for (int j = 0; j < CW; ++j)
#pragma unroll
              for (int i = 0; i < SWD; ++i)
                if (i < sw) cfms(v[j], a[q][i], S.Us[i * MAXNB + u0 + j]);
#pragma unroll
            for (int j = 0; j < CW; ++j)
              if (u0 + j < nright) arow[(size_t)(u0 + j) * N] = v[j];
          }
        }
      }
    }
    __syncthreads();
  }
  if (t == 0) info_all[b] = S.s_info;
}

// ---------------------------------------------------------------------------
// Inverses of the diagonal block: strictly-lower part -> unit-lower inverse
// (columns right to left), upper part -> upper inverse (columns left to right),
// both in place in shared memory as LAPACK's xTRTI2 does.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256)
k_triinv(const T *M, size_t strideM, int N, int J, int jb, int NB, int nsteps, T *Linv, T *Uinv,
         const int *ipiv_all, int *rmap_all) {
  extern __shared__ __align__(16) unsigned char smraw[];
  T *D = reinterpret_cast<T *>(smraw);
  T *tmp = D + NB * NB;
  __shared__ T s_d;
  __shared__ int keys[2 * MAXNB], content[2 * MAXNB];
  const int b = blockIdx.x, t = threadIdx.x, nt = blockDim.x;
  const T *A = M + (size_t)b * strideM;
  const int n = jb;
  if (t == 0) {
    // compose the step's interchanges (row J+i <-> ipiv[J+i], in order) into
    // one map over the rows they touch
    const int *ip = ipiv_all + (size_t)b * N + J;
    int nk = jb;
    for (int i = 0; i < jb; ++i) { keys[i] = J + i; content[i] = J + i; }
    for (int i = 0; i < jb; ++i) {
      const int p = ip[i];
      if (p == J + i) continue;
      int k;
      if (p < J + jb) {
        k = p - J;
      } else {
        k = -1;
        for (int q = jb; q < nk; ++q)
          if (keys[q] == p) { k = q; break; }
        if (k < 0) { k = nk++; keys[k] = p; content[k] = p; }
      }
      const int x = content[i]; content[i] = content[k]; content[k] = x;
    }
    int *rm = rmap_all + (size_t)b * RMAP_STRIDE;
    int cnt = 0;
    for (int k = 0; k < nk; ++k)
      if (content[k] != keys[k]) { rm[1 + 2 * cnt] = keys[k]; rm[2 + 2 * cnt] = content[k]; ++cnt; }
    rm[0] = cnt;
  }
  for (int e = t; e < n * n; e += nt) {
    int i = e % n, j = e / n;
    D[i + j * NB] = A[(size_t)(J + i) + (size_t)(J + j) * N];
  }
  __syncthreads();
  for (int j = n - 2; j >= 0; --j) {
    for (int i = j + 1 + t; i < n; i += nt) tmp[i] = D[i + j * NB];
    __syncthreads();
    for (int i = j + 1 + t; i < n; i += nt) {
      T s = tmp[i];
      for (int k = j + 1; k < i; ++k) cfma(s, D[i + k * NB], tmp[k]);
      D[i + j * NB] = cneg(s);
    }
    __syncthreads();
  }
  for (int j = 0; j < n; ++j) {
    if (t == 0) { T d = crcp(D[j + j * NB]); D[j + j * NB] = d; s_d = d; }
    for (int i = t; i < j; i += nt) tmp[i] = D[i + j * NB];
    __syncthreads();
    const T d = s_d;
    for (int i = t; i < j; i += nt) {
      T s = czero<T>();
      for (int k = i; k < j; ++k) cfma(s, D[i + k * NB], tmp[k]);
      D[i + j * NB] = cneg(cmul(d, s));
    }
    __syncthreads();
  }
  const size_t off = ((size_t)b * nsteps + J / NB) * NB * NB;
  for (int e = t; e < NB * NB; e += nt) {
    int i = e % NB, k = e / NB;
    T lv = czero<T>(), uv = czero<T>();
    if (i < n && k < n) {
      if (i > k) lv = D[i + k * NB];
      else if (i == k) lv = cx<T>::make(1, 0);
      if (i <= k) uv = D[i + k * NB];
    }
    Linv[off + e] = lv;
    Uinv[off + e] = uv;
  }
}

// ---------------------------------------------------------------------------
// Row interchanges of one step on the columns outside the panel, then
// U12 = L11^-1 A12 on the right columns (a jb x jb x TW product).
//
// The interchange map of the step (at most 2*NB <= 128 rows for NB <= 64) is
// applied to a TW-column tile with every load issued before a barrier and
// every store after it; thread (t % 64, t / 64) moves rows t%64 and t%64 + 64
// of columns t/64 + 4v.  Left tiles (columns left of the panel, needed by the
// forward solves) only swap rows and run in k_swap_left, which holds no
// dynamic shared memory.  A k_swap_trsm CTA stages L11^-1 (lower triangle,
// zero above) once and walks TPC column tiles: swap, stage the A12 tile,
// multiply.  Both operands are arranged so that the FP32 path uses packed
// two-lane FMAs (L as (re, re, -im, im), A12 as (re, im, im, re)).  Warp w
// owns row blocks w and 15 - w (4 rows each), so every warp does the same
// triangular k work; lane (r, cq) owns row r of each block and columns
// cq + 8n (n < 4).
// ---------------------------------------------------------------------------
#define TW 32
constexpr int TS_LD = 65;        // A12 tile column stride (elements) in shared memory
constexpr int TPC = 4;           // column tiles per k_swap_trsm CTA (L11^-1 staged once)

template <typename T>
__device__ __forceinline__ int load_map(const int *rm, int *s_map) {
  const int cnt = min(rm[0], 128);
  for (int i = threadIdx.x; i < 2 * cnt; i += 256) s_map[i] = rm[1 + i];
  return cnt;
}
// every load of the tile before a barrier, every store after it (s_map loaded and synced)
template <typename T>
__device__ __forceinline__ void swap_tile(T *A, int N, int cnt, int cs, int nc, const int *s_map) {
  const int t = threadIdx.x, kk = t & 63, cc = t >> 6;
  T v[2][8];
#pragma unroll
  for (int u = 0; u < 2; ++u)
#pragma unroll
    for (int w = 0; w < 8; ++w) {
      const int k = kk + 64 * u, c = cc + 4 * w;
      if (k < cnt && c < nc) v[u][w] = A[(size_t)s_map[2 * k + 1] + (size_t)(cs + c) * N];
    }
  __syncthreads();
#pragma unroll
  for (int u = 0; u < 2; ++u)
#pragma unroll
    for (int w = 0; w < 8; ++w) {
      const int k = kk + 64 * u, c = cc + 4 * w;
      if (k < cnt && c < nc) A[(size_t)s_map[2 * k] + (size_t)(cs + c) * N] = v[u][w];
    }
}

template <typename T>
__global__ void __launch_bounds__(256)
k_swap_left(T *M, size_t strideM, int N, int J, const int *rmap_all) {
  __shared__ int s_map[4 * 64];
  const int cs = blockIdx.x * TW, b = blockIdx.y;
  const int cnt = load_map<T>(rmap_all + (size_t)b * RMAP_STRIDE, s_map);
  __syncthreads();
  swap_tile<T>(M + (size_t)b * strideM, N, cnt, cs, min(J, cs + TW) - cs, s_map);
}

template <typename T> struct TrsmOp;
template <> struct TrsmOp<z32> {
  typedef float4 L;
  typedef float4 X;
  static __device__ __forceinline__ L packL(z32 l) { return make_float4(l.x, l.x, -l.y, l.y); }
  static __device__ __forceinline__ X packX(z32 x) { return make_float4(x.x, x.y, x.y, x.x); }
  static __device__ __forceinline__ void fma(z32 &acc, const L &l, const X &x) {
    acc = __ffma2_rn(make_float2(l.x, l.y), make_float2(x.x, x.y), acc);
    acc = __ffma2_rn(make_float2(l.z, l.w), make_float2(x.z, x.w), acc);
  }
};
template <> struct TrsmOp<z64> {
  typedef z64 L;
  typedef z64 X;
  static __device__ __forceinline__ L packL(z64 l) { return l; }
  static __device__ __forceinline__ X packX(z64 x) { return x; }
  static __device__ __forceinline__ void fma(z64 &acc, const L &l, const X &x) { cfma(acc, l, x); }
};

template <typename T>
__global__ void __launch_bounds__(256)
k_swap_trsm(T *M, size_t strideM, int N, int ncols, int J, int jb, int NB, int nsteps,
            const int *rmap_all, const T *Linv) {
  typedef TrsmOp<T> Op;
  extern __shared__ __align__(16) unsigned char smraw[];
  typename Op::L *Ls = reinterpret_cast<typename Op::L *>(smraw);           // [64 k][64 i]
  typename Op::X *Xs = reinterpret_cast<typename Op::X *>(Ls + 64 * 64);    // [TW c][TS_LD k]
  __shared__ int s_map[4 * 64];
  const int b = blockIdx.y, t = threadIdx.x;
  T *A = M + (size_t)b * strideM;
  const T *L = Linv + ((size_t)b * nsteps + J / NB) * NB * NB;
  for (int e = t; e < 64 * 64; e += 256) {
    const int i = e & 63, k = e >> 6;
    Ls[e] = Op::packL((i < jb && k <= i) ? L[i + k * NB] : czero<T>());
  }
  const int cnt = load_map<T>(rmap_all + (size_t)b * RMAP_STRIDE, s_map);
  // warp w owns row blocks w and 15-w (4 rows each): equal k work per warp
  const int warp = t >> 5, lane = t & 31, r = lane & 3, cq = lane >> 2;
  const int ia = 4 * warp + r, ib = 4 * (15 - warp) + r;
  const int ka = min(4 * warp + 4, jb), kb = min(4 * (16 - warp), jb);
  for (int tile = 0; tile < TPC; ++tile) {
    const int cs = J + jb + (blockIdx.x * TPC + tile) * TW;
    if (cs >= ncols) break;
    const int nc = min(ncols, cs + TW) - cs;
    __syncthreads();               // map and L staged; the previous tile's Xs reads are done
    swap_tile<T>(A, N, cnt, cs, nc, s_map);
    __syncthreads();
    for (int e = t; e < 64 * TW; e += 256) {
      const int k = e & 63, c = e >> 6;
      Xs[k + c * TS_LD] =
          Op::packX((k < jb && c < nc) ? A[(size_t)(J + k) + (size_t)(cs + c) * N] : czero<T>());
    }
    __syncthreads();
    T acc[2][4];
#pragma unroll
    for (int m = 0; m < 2; ++m)
#pragma unroll
      for (int n = 0; n < 4; ++n) acc[m][n] = czero<T>();
    int k = 0;
#pragma unroll 2
    for (; k < ka; ++k) {
      const typename Op::L la = Ls[ia + k * 64], lb = Ls[ib + k * 64];
#pragma unroll
      for (int n = 0; n < 4; ++n) {
        const typename Op::X x = Xs[k + (cq + 8 * n) * TS_LD];
        Op::fma(acc[0][n], la, x);
        Op::fma(acc[1][n], lb, x);
      }
    }
#pragma unroll 2
    for (; k < kb; ++k) {
      const typename Op::L lb = Ls[ib + k * 64];
#pragma unroll
      for (int n = 0; n < 4; ++n) Op::fma(acc[1][n], lb, Xs[k + (cq + 8 * n) * TS_LD]);
    }
#pragma unroll
    for (int m = 0; m < 2; ++m) {
      const int i = m ? ib : ia;
      if (i < jb)
#pragma unroll
        for (int n = 0; n < 4; ++n) {
          const int c = cq + 8 * n;
          if (c < nc) A[(size_t)(J + i) + (size_t)(cs + c) * N] = acc[m][n];
        }
    }
  }
}

// ---------------------------------------------------------------------------
// Unpivoted step (the FP32 factorisation of the mixed path, a preconditioner
// of the FP64 refinement): the BSE matrices are close to the identity (growth
// factor 1.00 and condition numbers of 1..40 on the t2g workload), so the
// factorisation needs no row interchanges.  Per step:
//   k_diag_inv    LU of the jb x jb diagonal block in shared memory with its
//                 inverted L11 / U11 blocks (one CTA per matrix); identity
//                 pivots and an empty interchange map;
//   k_tri_tile    L21 = A21 U11^-1 and U12 = L11^-1 A12, every row / column
//                 independent (no pivot search over the column).
// A zero pivot gives non-finite factors; the refinement then fails to
// converge and the point is re-solved in FP64 with partial pivoting.
// ---------------------------------------------------------------------------
constexpr int DN_LD = 65;

// Diagonal block of an unpivoted step with its inverses, one CTA per matrix
// (FP32): the jb x jb block is padded with the identity to 64 x 64 and
// factored right-looking in 4 x 4 register blocks, loaded straight from the
// matrix (16 block steps, two barriers each, packed two-lane FMAs in the
// trailing blocks; the next step's diagonal block is factored by its owner
// right after its own trailing update, so that factorisation overlaps the
// other blocks' updates).  L11^-1 (strictly lower; unit diagonal implied) and
// U11^-1 (upper with the diagonal) then share one array: eight warps invert
// the 16 x 16 diagonal blocks of both triangles (lane = column, no barriers),
// and two levels of recursive doubling join them,
//   [X00 0; X10 X11] with X10 = -X11 (L10 X00)   (and the transposed form for U),
// 16 x 16 blocks, then 32 x 32 blocks, the products L10 X00 formed in place of
// L10 (the factored block goes to the matrix before the inversion).  73 KB of
// shared memory: three CTAs per SM.
constexpr int DI_SCR = 3 * 256;

__device__ __forceinline__ void cfma2(z32 &acc, z32 a, z32 u) {
  acc = __ffma2_rn(make_float2(a.x, a.x), u, acc);
  acc = __ffma2_rn(make_float2(-a.y, a.y), make_float2(u.y, u.x), acc);
}
__device__ __forceinline__ void cfma2(z64 &acc, z64 a, z64 u) { cfma(acc, a, u); }
// 1 / z for the FP32 block LU: z = s (a + i b) with s = max(|Re z|, |Im z|), so that
// a^2 + b^2 lies in [1, 2]; two correctly rounded reciprocals (a zero pivot gives
// non-finite factors, which the refinement reports)
__device__ __forceinline__ z32 crcp_lu(z32 z) {
  const float is = __frcp_rn(fmaxf(fabsf(z.x), fabsf(z.y)));
  const float a = z.x * is, b = z.y * is;
  const float f = __frcp_rn(fmaf(a, a, b * b)) * is;
  return make_float2(a * f, -b * f);
}

template <typename T>
__global__ void __launch_bounds__(256, 3)
k_diag_inv(T *M, size_t strideM, int N, int J, int jb, int NB, int nsteps, T *Linv, T *Uinv, int *ipiv_all,
           int *rmap_all) {
  static_assert(sizeof(T) == sizeof(z32), "the blocked LU is the FP32 path's");
  extern __shared__ __align__(16) unsigned char smraw[];
  T *D = reinterpret_cast<T *>(smraw);          // [64][DN_LD] factored block
  T *X = D + 64 * DN_LD;                        // L11^-1 below the diagonal, U11^-1 on and above it
  T *S = X + 64 * DN_LD;                        // the LU's panel exchange
  __shared__ T rcps[64];
  const int b = blockIdx.x, t = threadIdx.x;
  T *A = M + (size_t)b * strideM;
  const T one = cx<T>::make(1, 0), zero = czero<T>();
  const int bi = t >> 4, bj = t & 15;
  T a[4][4];
  {
    // thread (bi, bj) owns D[4bi.., 4bj..]: four 32-byte column pieces, all loads in flight
#pragma unroll
    for (int c = 0; c < 4; ++c)
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const int i = 4 * bi + r, j = 4 * bj + c;
        a[r][c] = (i < jb && j < jb) ? A[(size_t)(J + i) + (size_t)(J + j) * N] : (i == j ? one : zero);
      }
  }
  {
    // Right-looking LU in 4 x 4 blocks.  Per block step kb: the owner of the diagonal block
    // has factored it (unit L, U, the reciprocals of U's diagonal) into xD; the column panel
    // solves L[bi,kb] U_kk = A[bi,kb], the row panel L_kk U[kb,bj] = A[kb,bj]; the trailing
    // blocks take A -= L[bi,kb] U[kb,bj] as four rank-1 updates, and the owner of block
    // (kb + 1, kb + 1) then factors it.  Panels are exchanged through S (stride 17 per
    // block, conflict-free for the 16 column owners of a warp).
    T *xL = S, *xU = S + 16 * 17, *xD = S + 2 * 16 * 17;   // xD: the factored diagonal block + 1/u
    auto factor_diag = [&](int kb) {
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const T rp = crcp_lu(a[k][k]);
        xD[16 + k] = rp;
        rcps[4 * kb + k] = rp;
#pragma unroll
        for (int i = k + 1; i < 4; ++i) a[i][k] = cmul(a[i][k], rp);
#pragma unroll
        for (int i = k + 1; i < 4; ++i)
#pragma unroll
          for (int j = k + 1; j < 4; ++j) a[i][j] = csub(a[i][j], cmul(a[i][k], a[k][j]));
      }
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) xD[r + 4 * c] = a[r][c];
    };
    if (t == 0) factor_diag(0);
    __syncthreads();
#pragma unroll 1
    for (int kb = 0; kb < 16; ++kb) {
      if (bj == kb && bi > kb) {
        // L[bi,kb] = A[bi,kb] U_kk^-1, column by column
#pragma unroll
        for (int c = 0; c < 4; ++c)
#pragma unroll
          for (int r = 0; r < 4; ++r) {
            T v = a[r][c];
#pragma unroll
            for (int c2 = 0; c2 < c; ++c2) v = csub(v, cmul(a[r][c2], xD[c2 + 4 * c]));
            a[r][c] = cmul(v, xD[16 + c]);
          }
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
          for (int c = 0; c < 4; ++c) xL[bi * 17 + r + 4 * c] = a[r][c];
      } else if (bi == kb && bj > kb) {
        // U[kb,bj] = L_kk^-1 A[kb,bj] (unit diagonal), row by row
#pragma unroll
        for (int r = 1; r < 4; ++r)
#pragma unroll
          for (int c = 0; c < 4; ++c)
#pragma unroll
            for (int r2 = 0; r2 < r; ++r2) a[r][c] = csub(a[r][c], cmul(xD[r + 4 * r2], a[r2][c]));
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
          for (int c = 0; c < 4; ++c) xU[bj * 17 + r + 4 * c] = a[r][c];
      }
      __syncthreads();
      if (bi > kb && bj > kb) {
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          T l[4], u[4];
#pragma unroll
          for (int r = 0; r < 4; ++r) l[r] = xL[bi * 17 + r + 4 * k];
#pragma unroll
          for (int c = 0; c < 4; ++c) u[c] = xU[bj * 17 + k + 4 * c];
          // a[r][c] -= l[r] u[c] as two packed FMAs per complex entry
#pragma unroll
          for (int c = 0; c < 4; ++c) {
            const float2 us = make_float2(u[c].y, u[c].x);
#pragma unroll
            for (int r = 0; r < 4; ++r) {
              a[r][c] = __ffma2_rn(make_float2(-l[r].x, -l[r].x), u[c], a[r][c]);
              a[r][c] = __ffma2_rn(make_float2(l[r].y, -l[r].y), us, a[r][c]);
            }
          }
        }
        // xD is free once the panels are solved: the next diagonal block is factored now
        if (bi == kb + 1 && bj == kb + 1) factor_diag(kb + 1);
      }
      __syncthreads();
    }
    // the packed factors (multipliers below the diagonal, U on and above it) into D and the matrix
#pragma unroll
    for (int c = 0; c < 4; ++c)
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const int i = 4 * bi + r, j = 4 * bj + c;
        D[i + j * DN_LD] = a[r][c];
        if (i < jb && j < jb) A[(size_t)(J + i) + (size_t)(J + j) * N] = a[r][c];
      }
  }
  __syncthreads();
  // entries of the two inverses: L^-1 with its unit diagonal and zeros above, U^-1 with zeros below
  auto xl = [&](int r, int c) { return r > c ? X[r + c * DN_LD] : (r == c ? one : zero); };
  auto xu = [&](int r, int c) { return r <= c ? X[r + c * DN_LD] : zero; };
  {
    // the 16 x 16 diagonal blocks of both inverses: warp w < 4 column l of L block w, warp w >= 4
    // column l of U block w - 4, by substitution
    const int w = t >> 5, lane = t & 31;
    if (lane < 16) {
      const int o = 16 * (w & 3), l = lane;
      T x[16];
      const T xd = w < 4 ? one : rcps[o + l];    // diagonal entry of the inverse's column l
#pragma unroll
      for (int r = 0; r < 16; ++r) x[r] = r == l ? xd : zero;
      if (w < 4) {                                // unit lower: column l of the block inverse, below l
#pragma unroll
        for (int r = 1; r < 16; ++r) {
          if (r > l) {
            T s = zero;
#pragma unroll
            for (int kk = 0; kk < r; ++kk)
              if (kk >= l) cfma(s, D[(o + r) + (o + kk) * DN_LD], x[kk]);
            x[r] = cneg(s);
          }
        }
#pragma unroll
        for (int r = 0; r < 16; ++r)
          if (r > l) X[(o + r) + (o + l) * DN_LD] = x[r];
      } else {                                    // upper: column l, on and above the diagonal
#pragma unroll
        for (int r = 14; r >= 0; --r) {
          if (r < l) {
            T s = zero;
#pragma unroll
            for (int kk = r + 1; kk < 16; ++kk)
              if (kk <= l) cfma(s, D[(o + r) + (o + kk) * DN_LD], x[kk]);
            x[r] = cneg(cmul(rcps[o + r], s));
          }
        }
#pragma unroll
        for (int r = 0; r < 16; ++r)
          if (r <= l) X[(o + r) + (o + l) * DN_LD] = x[r];
      }
    }
  }
  __syncthreads();
  {
    // 16 -> 32: for the 32-blocks at o = 0, 32 of both triangles
    //   L: X10 = -X11 (L10 X00),   U: Y01 = -Y00 (U01 Y11),
    // warp w: product (w >> 1): L at o = 0, 32, then U at o = 0, 32; columns 8 (w & 1).. + 7;
    // lane: row i = lane & 15, columns 4 (lane >> 4) + q
    const int w = t >> 5, lane = t & 31;
    const bool up = w >= 4;
    const int o = 32 * ((w >> 1) & 1), i = lane & 15, j0 = 8 * (w & 1) + 4 * (lane >> 4);
    T v[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) v[q] = zero;
    if (!up) {
#pragma unroll 4
      for (int k = 0; k < 16; ++k) {
        const T d = D[(o + 16 + i) + (o + k) * DN_LD];
#pragma unroll
        for (int q = 0; q < 4; ++q) cfma2(v[q], d, xl(o + k, o + j0 + q));
      }
    } else {
#pragma unroll 4
      for (int k = 0; k < 16; ++k) {
        const T d = D[(o + i) + (o + 16 + k) * DN_LD];
#pragma unroll
        for (int q = 0; q < 4; ++q) cfma2(v[q], d, xu(o + 16 + k, o + 16 + j0 + q));
      }
    }
    __syncthreads();     // every product has read its block of D: the products replace them
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      if (!up) D[(o + 16 + i) + (o + j0 + q) * DN_LD] = v[q];
      else D[(o + i) + (o + 16 + j0 + q) * DN_LD] = v[q];
      v[q] = zero;
    }
    __syncthreads();
    if (!up) {
#pragma unroll 4
      for (int k = 0; k < 16; ++k) {
        const T x = xl(o + 16 + i, o + 16 + k);
#pragma unroll
        for (int q = 0; q < 4; ++q) cfma2(v[q], x, D[(o + 16 + k) + (o + j0 + q) * DN_LD]);
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) X[(o + 16 + i) + (o + j0 + q) * DN_LD] = cneg(v[q]);
    } else {
#pragma unroll 4
      for (int k = 0; k < 16; ++k) {
        const T x = xu(o + i, o + k);
#pragma unroll
        for (int q = 0; q < 4; ++q) cfma2(v[q], x, D[(o + k) + (o + 16 + j0 + q) * DN_LD]);
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) X[(o + i) + (o + 16 + j0 + q) * DN_LD] = cneg(v[q]);
    }
  }
  __syncthreads();
  {
    // 32 -> 64: L: X10 = -X11 (L10 X00), U: Y01 = -Y00 (U01 Y11) with 32 x 32 blocks;
    // warp w: columns 4w + q of both products, lane: row i
    const int w = t >> 5, i = t & 31, j0 = 4 * w;
    T vl[4], vu[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) vl[q] = vu[q] = zero;
    // L10 X00: X00(k, j) = 0 for k < j
#pragma unroll 4
    for (int k = j0; k < 32; ++k) {
      const T d = D[(32 + i) + k * DN_LD];
#pragma unroll
      for (int q = 0; q < 4; ++q) cfma2(vl[q], d, xl(k, j0 + q));
    }
    // U01 Y11: Y11(k, j) = 0 for k > j
#pragma unroll 4
    for (int k = 0; k < j0 + 4; ++k) {
      const T d = D[i + (32 + k) * DN_LD];
#pragma unroll
      for (int q = 0; q < 4; ++q) cfma2(vu[q], d, xu(32 + k, 32 + j0 + q));
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      D[(32 + i) + (j0 + q) * DN_LD] = vl[q];
      D[i + (32 + j0 + q) * DN_LD] = vu[q];
      vl[q] = vu[q] = zero;
    }
    __syncthreads();
#pragma unroll 4
    for (int k = 0; k < 32; ++k) {
      const T xa = xl(32 + i, 32 + k), xb = xu(i, k);
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        cfma2(vl[q], xa, D[(32 + k) + (j0 + q) * DN_LD]);
        cfma2(vu[q], xb, D[k + (32 + j0 + q) * DN_LD]);
      }
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      X[(32 + i) + (j0 + q) * DN_LD] = cneg(vl[q]);
      X[i + (32 + j0 + q) * DN_LD] = cneg(vu[q]);
    }
  }
  __syncthreads();
  const size_t off = ((size_t)b * nsteps + J / NB) * NB * NB;
#pragma unroll 4
  for (int e = t; e < NB * NB; e += 256) {
    const int i = e % NB, k = e / NB;
    T lv = zero, uv = zero;
    if (i < jb && k < jb) {
      lv = xl(i, k);
      uv = xu(i, k);
    }
    Linv[off + e] = lv;
    Uinv[off + e] = uv;
  }
  int *ip = ipiv_all + (size_t)b * N + J;
  for (int i = t; i < jb; i += 256) ip[i] = J + i;
  if (t == 0) rmap_all[(size_t)b * RMAP_STRIDE] = 0;
}

// Off-diagonal tiles of an unpivoted step, 64 x 64 per CTA:
//   LEFT  U12 = L11^-1 A12  (rows J.., columns J+jb+64 x)
//   !LEFT L21 = A21 U11^-1  (rows J+jb+64 x.., columns J..)
// The tile and the triangle are staged in shared memory (column stride 65,
// conflict-free).  Along the triangle's free index (rows of U12, columns of
// L21) a thread owns 4 consecutive entries and the other index strides by
// 16; that index's owner, (t / 16), is nearly warp-uniform, so each warp
// stops at its own edge of the triangle and the product does the triangular
// half of the work.  U12 is written back through shared memory (coalesced).
// one element global -> shared by cp.async (8 or 16 bytes); zeros when !valid
template <typename T>
__device__ __forceinline__ void cp_async_elem(T *dst, const T *src, bool valid) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  if constexpr (sizeof(T) == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(d), "l"(src), "r"(valid ? 8 : 0));
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(src), "r"(valid ? 16 : 0));
}

template <typename T, bool LEFT>
__global__ void __launch_bounds__(256)
k_tri_tile(T *M, size_t strideM, int N, int ncols, int J, int jb, int NB, int nsteps, const T *Tri) {
  extern __shared__ __align__(16) unsigned char smraw[];
  T *Ts = reinterpret_cast<T *>(smraw);        // triangle, [k or row][DN_LD]
  T *Xs = Ts + 64 * DN_LD;                      // tile
  const int b = blockIdx.y, t = threadIdx.x;
  T *A = M + (size_t)b * strideM;
  const T *Q = Tri + ((size_t)b * nsteps + J / NB) * NB * NB;
  const int r0 = LEFT ? J : J + jb + blockIdx.x * 64;
  const int c0 = LEFT ? J + jb + blockIdx.x * 64 : J;
  const int nr = LEFT ? jb : min(64, N - r0);
  const int nc = LEFT ? min(64, ncols - c0) : jb;
  // asynchronous staging (zero-filled outside the triangle / tile): every load in flight at once
  for (int e = t; e < 64 * 64; e += 256) {
    const int i = e & 63, j = e >> 6;           // i fastest: coalesced loads, conflict-free stores
    const bool inq = i < jb && j < jb, inx = i < nr && j < nc;
    cp_async_elem<T>(Ts + i + j * DN_LD, inq ? Q + i + (size_t)j * NB : Q, inq);
    cp_async_elem<T>(Xs + i + j * DN_LD, inx ? A + (size_t)(r0 + i) + (size_t)(c0 + j) * N : A, inx);
  }
  asm volatile("cp.async.commit_group;");
  asm volatile("cp.async.wait_group 0;" ::: "memory");
  __syncthreads();
  const int w4 = 4 * (t >> 4), s16 = t & 15;    // 4 consecutive triangle-side entries, the rest by 16
  T acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = czero<T>();
  // LEFT: out(w4 + i, s16 + 16 j) = sum_{k <= row} L^-1(row, k) X(k, col)
  // !LEFT: out(s16 + 16 i, w4 + j) = sum_{k <= col} X(row, k) U^-1(k, col)
  const int kend = min(jb, w4 + 4);
#pragma unroll 2
  for (int k = 0; k < kend; ++k) {
    T a[4], u[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) a[i] = LEFT ? Ts[(w4 + i) + k * DN_LD] : Xs[(s16 + 16 * i) + k * DN_LD];
#pragma unroll
    for (int j = 0; j < 4; ++j) u[j] = LEFT ? Xs[k + (s16 + 16 * j) * DN_LD] : Ts[k + (w4 + j) * DN_LD];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) cfma2(acc[i][j], a[i], u[j]);
  }
  if (LEFT) {
    __syncthreads();                            // every Xs read is done
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) Xs[(w4 + i) + (s16 + 16 * j) * DN_LD] = acc[i][j];
    __syncthreads();
    for (int e = t; e < 64 * 64; e += 256) {
      const int i = e & 63, j = e >> 6;
      if (i < nr && j < nc) A[(size_t)(r0 + i) + (size_t)(c0 + j) * N] = Xs[i + j * DN_LD];
    }
  } else {
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int c = w4 + j;
      if (c >= nc) continue;
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int r = s16 + 16 * i;
        if (r < nr) A[(size_t)(r0 + r) + (size_t)(c0 + c) * N] = acc[i][j];
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Trailing update on CUDA cores: C[J+jb.., J+jb..] -= A[J+jb.., J:J+jb] * A[J:J+jb, J+jb..]
// 64 x 64 tiles, BK = 16, 256 threads with 4 x 4 complex outputs each.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256)
k_gemm_update(T *M, size_t strideM, int N, int ncols, int J, int jb) {
  __shared__ T As[16][64];
  __shared__ T Bs[16][64];
  const int b = blockIdx.z, t = threadIdx.x;
  const int tx = t & 15, ty = t >> 4;
  T *A = M + (size_t)b * strideM;
  const int r0 = J + jb + blockIdx.y * 64, c0 = J + jb + blockIdx.x * 64;
  T acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = czero<T>();
  for (int k0 = 0; k0 < jb; k0 += 16) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      int e = t + 256 * i;
      int rr = e & 63, kk = e >> 6;
      int r = r0 + rr, k = k0 + kk;
      As[kk][rr] = (r < N && k < jb) ? A[r + (size_t)(J + k) * N] : czero<T>();
      int kk2 = e & 15, cc = e >> 4;
      int c = c0 + cc, k2 = k0 + kk2;
      Bs[kk2][cc] = (c < ncols && k2 < jb) ? A[(size_t)(J + k2) + (size_t)c * N] : czero<T>();
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < 16; ++kk) {
      T av[4], bv[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) av[i] = As[kk][tx + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; ++j) bv[j] = Bs[kk][ty + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) cfma(acc[i][j], av[i], bv[j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int c = c0 + ty + 16 * j;
    if (c >= ncols) continue;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int r = r0 + tx + 16 * i;
      if (r < N) {
        T *p = A + r + (size_t)c * N;
        *p = csub(*p, acc[i][j]);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Blocked triangular solves with the inverted diagonal blocks.
// backsolve: U Y = C (bottom block first); fwdsolve: L z = P r (top first).
// ---------------------------------------------------------------------------
#define RT 16
template <typename T, bool UPPER>
__global__ void __launch_bounds__(256)
k_trisolve(const T *M, size_t strideM, int N, int NB, int nsteps, const T *Dinv, T *C,
           size_t strideC, int ldc, int R, const int *ipiv_all, T *work) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const int nph = 256 / NB;
  T *red = reinterpret_cast<T *>(smraw);          // [nph][NB][RT]
  T *W = red + (size_t)nph * NB * RT;             // [NB][RT]
  int *perm = reinterpret_cast<int *>(W + (size_t)NB * RT);
  const int b = blockIdx.y, r0 = blockIdx.x * RT, t = threadIdx.x;
  const T *A = M + (size_t)b * strideM;
  T *Cb = C + (size_t)b * strideC;
  const int nr = min(RT, R - r0);
  if (!UPPER) {
    // apply the row interchanges P to the right-hand sides (through work)
    if (t == 0) {
      for (int i = 0; i < N; ++i) perm[i] = i;
      const int *ip = ipiv_all + (size_t)b * N;
      for (int i = 0; i < N; ++i) {
        int p = ip[i];
        if (p != i) { int x = perm[i]; perm[i] = perm[p]; perm[p] = x; }
      }
    }
    __syncthreads();
    T *Wk = work + (size_t)b * N * RT * gridDim.x + (size_t)blockIdx.x * N * RT;
    for (int e = t; e < N * nr; e += 256) {
      int i = e % N, r = e / N;
      Wk[e] = Cb[perm[i] + (size_t)(r0 + r) * ldc];
    }
    __syncthreads();
    for (int e = t; e < N * nr; e += 256) {
      int i = e % N, r = e / N;
      Cb[i + (size_t)(r0 + r) * ldc] = Wk[e];
    }
    __syncthreads();
  }
  const int row = t % NB, kph = t / NB;
  for (int s = 0; s < nsteps; ++s) {
    const int blk = UPPER ? nsteps - 1 - s : s;
    const int J = blk * NB, jb = min(NB, N - J);
    T acc[RT];
#pragma unroll
    for (int r = 0; r < RT; ++r) acc[r] = czero<T>();
    if (row < jb) {
      const int kb = UPPER ? J + jb : 0, ke = UPPER ? N : J;
      for (int k = kb + kph; k < ke; k += nph) {
        const T u = A[(size_t)(J + row) + (size_t)k * N];
#pragma unroll
        for (int r = 0; r < RT; ++r)
          if (r < nr) cfma(acc[r], u, Cb[k + (size_t)(r0 + r) * ldc]);
      }
    }
#pragma unroll
    for (int r = 0; r < RT; ++r) red[((size_t)kph * NB + row) * RT + r] = acc[r];
    __syncthreads();
    for (int e = t; e < jb * nr; e += 256) {
      int i = e % jb, r = e / jb;
      T v = Cb[(size_t)(J + i) + (size_t)(r0 + r) * ldc];
      for (int ph = 0; ph < nph; ++ph) v = csub(v, red[((size_t)ph * NB + i) * RT + r]);
      W[i * RT + r] = v;
    }
    __syncthreads();
    const T *Di = Dinv + ((size_t)b * nsteps + blk) * NB * NB;
    for (int e = t; e < jb * nr; e += 256) {
      int i = e % jb, r = e / jb;
      T v = czero<T>();
      const int kb = UPPER ? i : 0, ke = UPPER ? jb : i + 1;
      for (int k = kb; k < ke; ++k) cfma(v, Di[i + k * NB], W[k * RT + r]);
      Cb[(size_t)(J + i) + (size_t)(r0 + r) * ldc] = v;
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Blocked triangular solve with the right-hand sides resident in shared
// memory (R <= RMAX columns, N*R elements): one CTA per matrix, right-looking
// over the NB-row blocks.  Per block: X_blk = Dinv * C_blk, then the rows not
// yet solved are updated with the matching column block of U (backward) or L
// (forward), one thread per row, so every element of the triangle is read
// from HBM exactly once with coalesced column accesses.  The forward solve
// applies the row interchanges P while loading the right-hand sides.
// ---------------------------------------------------------------------------
template <typename T, bool UPPER, int RMAX, int RPT>
__global__ void __launch_bounds__(512)
k_trisolve_smem(const T *M, size_t strideM, int N, int NB, int nsteps, const T *Dinv, T *C,
                size_t strideC, int ldc, int R, const int *ipiv_all, size_t stage_d) {
  extern __shared__ __align__(16) unsigned char smraw[];
  T *Cs = reinterpret_cast<T *>(smraw);            // [R][N]
  T *Yt = Cs + (size_t)N * R;                        // [R][NB]
  int *perm = reinterpret_cast<int *>(Yt + (size_t)NB * R);
  // the diagonal-block inverse of the current step, staged when it fits
  T *Ds = stage_d ? reinterpret_cast<T *>(smraw + stage_d) : nullptr;
  const int b = blockIdx.x, t = threadIdx.x, nt = blockDim.x;
  const T *A = M + (size_t)b * strideM;
  T *Cb = C + (size_t)b * strideC;
  if (!UPPER) {
    if (t == 0) {
      for (int i = 0; i < N; ++i) perm[i] = i;
      const int *ip = ipiv_all + (size_t)b * N;
      for (int i = 0; i < N; ++i) {
        const int p = ip[i];
        if (p != i) { int x = perm[i]; perm[i] = perm[p]; perm[p] = x; }
      }
    }
    __syncthreads();
  }
  for (int e = t; e < N * R; e += nt) {
    const int i = e % N, r = e / N;
    Cs[e] = Cb[(size_t)(UPPER ? i : perm[i]) + (size_t)r * ldc];
  }
  __syncthreads();
  for (int s = 0; s < nsteps; ++s) {
    const int blk = UPPER ? nsteps - 1 - s : s;
    const int J = blk * NB, jb = min(NB, N - J);
    const T *Di = Dinv + ((size_t)b * nsteps + blk) * NB * NB;
    if (Ds) {
      for (int e = t; e < NB * jb; e += nt) Ds[e] = Di[e];
      __syncthreads();
    }
    const T *D = Ds ? Ds : Di;
    for (int e = t; e < jb * R; e += nt) {
      const int i = e % jb, r = e / jb;
      const int kb = UPPER ? i : 0, ke = UPPER ? jb : i + 1;
      T v0 = czero<T>(), v1 = czero<T>(), v2 = czero<T>(), v3 = czero<T>();
      int k = kb;
      for (; k + 3 < ke; k += 4) {
        cfma(v0, D[i + k * NB], Cs[(size_t)r * N + J + k]);
        cfma(v1, D[i + (k + 1) * NB], Cs[(size_t)r * N + J + k + 1]);
        cfma(v2, D[i + (k + 2) * NB], Cs[(size_t)r * N + J + k + 2]);
        cfma(v3, D[i + (k + 3) * NB], Cs[(size_t)r * N + J + k + 3]);
      }
      for (; k < ke; ++k) cfma(v0, D[i + k * NB], Cs[(size_t)r * N + J + k]);
      Yt[(size_t)r * NB + i] = cadd(cadd(v0, v1), cadd(v2, v3));
    }
    __syncthreads();
    for (int e = t; e < jb * R; e += nt) {
      const int i = e % jb, r = e / jb;
      Cs[(size_t)r * N + J + i] = Yt[(size_t)r * NB + i];
    }
    // rows still to solve: each thread owns RPT of them, so every Yt value
    // read from shared memory feeds RPT rows
    const int rb = UPPER ? 0 : J + jb, re = UPPER ? J : N;
    for (int base = rb + t; base < re; base += nt * RPT) {
      T acc[RPT][RMAX];
#pragma unroll
      for (int q = 0; q < RPT; ++q)
#pragma unroll
        for (int r = 0; r < RMAX; ++r) acc[q][r] = czero<T>();
#pragma unroll 8
      for (int k = 0; k < jb; ++k) {
        T y[RMAX];
#pragma unroll
        for (int r = 0; r < RMAX; ++r) y[r] = r < R ? Yt[(size_t)r * NB + k] : czero<T>();
#pragma unroll
        for (int q = 0; q < RPT; ++q) {
          const int i = base + q * nt;
          const T u = i < re ? A[(size_t)i + (size_t)(J + k) * N] : czero<T>();
#pragma unroll
          for (int r = 0; r < RMAX; ++r)
            if (r < R) cfma(acc[q][r], u, y[r]);
        }
      }
#pragma unroll
      for (int q = 0; q < RPT; ++q) {
        const int i = base + q * nt;
        if (i < re)
#pragma unroll
          for (int r = 0; r < RMAX; ++r)
            if (r < R) Cs[(size_t)r * N + i] = csub(Cs[(size_t)r * N + i], acc[q][r]);
      }
    }
    __syncthreads();
  }
  for (int e = t; e < N * R; e += nt) {
    const int i = e % N, r = e / N;
    Cb[(size_t)i + (size_t)r * ldc] = Cs[e];
  }
}

// ---------------------------------------------------------------------------
// host drivers
// ---------------------------------------------------------------------------
template <typename T>
static cudaError_t launch_panel(T *M, const LUBatch &lb, int J, int jb, cudaStream_t st) {
  const int rows = lb.N - J;
  auto nthreads = [&](int rpt) { int n = ((rows + rpt - 1) / rpt + 31) / 32 * 32; return n < 32 ? 32 : n; };
  const size_t dyn = sizeof(T) * (size_t)MAXNB * 2 * SWD;
  smem_limit(k_panel<T, 1>, 96 * 1024);
  smem_limit(k_panel<T, 2>, 96 * 1024);
  smem_limit(k_panel<T, 4>, 96 * 1024);
  smem_limit(k_panel<T, 8>, 96 * 1024);
  // fewer, fuller threads per CTA: more matrices resident per SM and cheaper
  // block-wide pivot reductions (FP32 rows cost half the registers of FP64)
  const bool f32 = sizeof(T) == sizeof(z32);
  if (rows <= (f32 ? 0 : 1024)) {
    k_panel<T, 1><<<lb.batch, nthreads(1), dyn, st>>>(M, lb.strideM, lb.N, J, jb, lb.ipiv, lb.info);
  } else if (rows <= (f32 ? 0 : 1280)) {
    k_panel<T, 2><<<lb.batch, nthreads(2), dyn, st>>>(M, lb.strideM, lb.N, J, jb, lb.ipiv, lb.info);
  } else if (rows <= 2048) {
    k_panel<T, 4><<<lb.batch, nthreads(4), dyn, st>>>(M, lb.strideM, lb.N, J, jb, lb.ipiv, lb.info);
  } else if (rows <= 4096) {
    k_panel<T, 8><<<lb.batch, nthreads(8), dyn, st>>>(M, lb.strideM, lb.N, J, jb, lb.ipiv, lb.info);
  } else {
    return cudaErrorInvalidValue;   // N > 4096 is not supported
  }
  return ADGA_LAUNCH_CHECK();
}

cudaError_t lu_trail_z64(z64 *M, const LUBatch &lb, int J, int jb, cudaStream_t st);

template <typename T>
cudaError_t lu_trail_cuda(T *M, const LUBatch &lb, int J, int jb, cudaStream_t st) {
  if constexpr (sizeof(T) == sizeof(z64)) return lu_trail_z64((z64 *)M, lb, J, jb, st);
  const int m = lb.N - J - jb, n = lb.ncols - J - jb;
  if (m <= 0 || n <= 0) return cudaSuccess;
  dim3 grid(cdiv_u(n, 64), cdiv_u(m, 64), lb.batch);
  k_gemm_update<T><<<grid, 256, 0, st>>>(M, lb.strideM, lb.N, lb.ncols, J, jb);
  return ADGA_LAUNCH_CHECK();
}

// trailing update of step (J, jb) through `trail` (or the CUDA-core GEMM), timed into tt
template <typename T>
static cudaError_t lu_trail_step(T *M, const LUBatch &lb, int J, int jb, trail_fn trail, void *trail_ctx,
                                 cudaStream_t st, TrailTiming *tt) {
  cudaError_t e;
  if (J + jb < lb.N) {
    cudaEvent_t ev0 = (tt && tt->ev) ? tt->ev[2 * tt->n] : nullptr;
    cudaEvent_t ev1 = (tt && tt->ev) ? tt->ev[2 * tt->n + 1] : nullptr;
    if (trail) {
      e = trail(trail_ctx, J, jb, st, ev0, ev1);
    } else {
      if (ev0) cudaEventRecord(ev0, st);
      e = lu_trail_cuda<T>(M, lb, J, jb, st);
      if (ev1) cudaEventRecord(ev1, st);
    }
    if (e != cudaSuccess) return e;
    if (tt && tt->ev) {
      const double m = lb.N - J - jb, n = lb.ncols - J - jb;
      tt->gflop += 8.0 * m * n * jb * lb.batch * 1e-9;
      tt->gbytes += (2.0 * sizeof(T) * m * n + sizeof(T) * (double)jb * (m + n)) * lb.batch * 1e-9;
      tt->n++;
    }
  }
  return cudaSuccess;
}

// kernels of one unpivoted FP32 step: block LU + inverses, L21, U12 (k_diag_inv, k_tri_tile;
// tiles = false: the block LU only)
static cudaError_t nopiv_step_kernels(z32 *M, const LUBatch &lb, int J, int jb, cudaStream_t st,
                                      bool tiles = true) {
  typedef z32 T;
  const int nsteps = lb.nsteps();
  cudaError_t e;
  const size_t sm_di = sizeof(T) * (2 * 64 * DN_LD + DI_SCR), sm_tt = sizeof(T) * 2 * 64 * DN_LD;
  smem_limit(k_diag_inv<T>, (int)sm_di);
  smem_limit(k_tri_tile<T, true>, (int)sm_tt);
  smem_limit(k_tri_tile<T, false>, (int)sm_tt);
  k_diag_inv<T><<<lb.batch, 256, sm_di, st>>>(M, lb.strideM, lb.N, J, jb, lb.NB, nsteps, (T *)lb.Linv,
                                              (T *)lb.Uinv, lb.ipiv, lb.rmap);
  if ((e = ADGA_LAUNCH_CHECK()) != cudaSuccess) return e;
  if (!tiles) return cudaSuccess;
  if (J + jb < lb.N) {
    k_tri_tile<T, false><<<dim3(cdiv_u(lb.N - J - jb, 64), lb.batch), 256, sm_tt, st>>>(
        M, lb.strideM, lb.N, lb.ncols, J, jb, lb.NB, nsteps, (const T *)lb.Uinv);
    if ((e = ADGA_LAUNCH_CHECK()) != cudaSuccess) return e;
  }
  if (lb.ncols > J + jb) {
    k_tri_tile<T, true><<<dim3(cdiv_u(lb.ncols - J - jb, 64), lb.batch), 256, sm_tt, st>>>(
        M, lb.strideM, lb.N, lb.ncols, J, jb, lb.NB, nsteps, (const T *)lb.Linv);
    if ((e = ADGA_LAUNCH_CHECK()) != cudaSuccess) return e;
  }
  return cudaSuccess;
}

static void trail_account(TrailTiming *tt, double m, double n, double k, int batch) {
  if (!tt || !tt->ev || m <= 0 || n <= 0) return;
  tt->gflop += 8.0 * m * n * k * batch * 1e-9;
  tt->gbytes += (2.0 * sizeof(z32) * m * n + sizeof(z32) * k * (m + n)) * batch * 1e-9;
}

// Unpivoted FP32 factorisation with delayed updates in groups of G = 2..4 steps: after
// step g < G - 1 of a group only the parts of the group's updates that step g + 1 reads
// (narrow), after its last step all G steps' updates of the rest at once (wide)
cudaError_t lu_factor_groups(z32 *M, const LUBatch &lb, const GroupOps &ops, cudaStream_t st, TrailTiming *tt) {
  if (ops.G < 2 || ops.G > 4) return cudaErrorInvalidValue;
  const int nsteps = lb.nsteps();
  int Js[4], jbs[4];
  for (int s = 0; s < nsteps; ++s) {
    const int J = s * lb.NB, jb = min(lb.NB, lb.N - J), g = s % ops.G;
    Js[g] = J;
    jbs[g] = jb;
    cudaError_t e = nopiv_step_kernels(M, lb, J, jb, st, ops.tri == nullptr);
    if (e == cudaSuccess && ops.tri) e = ops.tri(ops.ctx, J, jb, g, st);
    if (e != cudaSuccess) return e;
    if (J + jb >= lb.N) break;
    cudaEvent_t ev0 = (tt && tt->ev) ? tt->ev[2 * tt->n] : nullptr;
    cudaEvent_t ev1 = (tt && tt->ev) ? tt->ev[2 * tt->n + 1] : nullptr;
    const bool wide = g == ops.G - 1;
    e = ops.update(ops.ctx, g + 1, Js, jbs, wide, st, ev0, ev1);
    int K = 0;
    for (int i = 0; i <= g; ++i) K += jbs[i];
    const int R = J + jb;
    if (wide) {
      trail_account(tt, lb.N - R, lb.ncols - R, K, lb.batch);
    } else {
      const int jt = min(lb.NB, lb.N - R);
      trail_account(tt, lb.N - R, jt, K, lb.batch);
      trail_account(tt, jt, lb.ncols - R - jt, K, lb.batch);
    }
    if (e != cudaSuccess) return e;
    if (tt && tt->ev) tt->n++;
  }
  return cudaSuccess;
}

template <typename T>
cudaError_t lu_step(T *M, const LUBatch &lb, int s, bool apply_left, trail_fn trail, void *trail_ctx,
                    cudaStream_t st, TrailTiming *tt, bool nopiv) {
  if (lb.NB > 64 || lb.NB % SWD) return cudaErrorInvalidValue;   // k_swap_trsm covers NB <= 64
  const int nsteps = lb.nsteps();
  cudaError_t e;
  const size_t sm_tri = sizeof(T) * ((size_t)lb.NB * lb.NB + lb.NB);
  const size_t sm_trsm = sizeof(typename TrsmOp<T>::L) * 64 * 64 + sizeof(typename TrsmOp<T>::X) * TW * TS_LD;
  smem_limit(k_triinv<T>, 200 * 1024);
  smem_limit(k_swap_trsm<T>, 200 * 1024);
  const int J = s * lb.NB, jb = min(lb.NB, lb.N - J);
  if constexpr (sizeof(T) == sizeof(z32)) {
    if (nopiv) {
      if ((e = nopiv_step_kernels(M, lb, J, jb, st)) != cudaSuccess) return e;
      return lu_trail_step<T>(M, lb, J, jb, trail, trail_ctx, st, tt);
    }
  }
  if (nopiv) return cudaErrorInvalidValue;     // the unpivoted step is the FP32 factorisation only
  if ((e = launch_panel<T>(M, lb, J, jb, st)) != cudaSuccess) return e;
  k_triinv<T><<<lb.batch, 256, sm_tri, st>>>(M, lb.strideM, lb.N, J, jb, lb.NB, nsteps,
                                             (T *)lb.Linv, (T *)lb.Uinv, lb.ipiv, lb.rmap);
  if ((e = ADGA_LAUNCH_CHECK()) != cudaSuccess) return e;
  const int nleft = apply_left ? (J + TW - 1) / TW : 0;
  const int nright = (lb.ncols - J - jb + TW - 1) / TW;
  if (nleft > 0) {
    k_swap_left<T><<<dim3(nleft, lb.batch), 256, 0, st>>>(M, lb.strideM, lb.N, J, lb.rmap);
    if ((e = ADGA_LAUNCH_CHECK()) != cudaSuccess) return e;
  }
  if (nright > 0) {
    k_swap_trsm<T><<<dim3((nright + TPC - 1) / TPC, lb.batch), 256, sm_trsm, st>>>(M, lb.strideM, lb.N, lb.ncols, J, jb, lb.NB,
                                                                 nsteps, lb.rmap, (const T *)lb.Linv);
    if ((e = ADGA_LAUNCH_CHECK()) != cudaSuccess) return e;
  }
  return lu_trail_step<T>(M, lb, J, jb, trail, trail_ctx, st, tt);
}

template <typename T>
cudaError_t lu_factor(T *M, const LUBatch &lb, bool apply_left, trail_fn trail, void *trail_ctx,
                      cudaStream_t st, TrailTiming *tt, bool nopiv) {
  for (int s = 0; s < lb.nsteps(); ++s) {
    cudaError_t e = lu_step<T>(M, lb, s, apply_left, trail, trail_ctx, st, tt, nopiv);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

template <typename T>
static cudaError_t trisolve(const T *M, const LUBatch &lb, T *C, size_t strideC, int ldc, int R,
                            bool upper, T *work, cudaStream_t st) {
  // FP32 factors, up to 16 right-hand sides: the tensor-core solve (k_trsv_tc.cu)
  if constexpr (sizeof(T) == sizeof(z32))
    if (trsv_tc_supported(lb, R, upper))
      return launch_trsv_tc(reinterpret_cast<const z32 *>(M), lb, reinterpret_cast<z32 *>(C), strideC, ldc, R,
                            upper, st);
  // few right-hand sides and NB = 64: the streaming solve (k_trsv.cu)
  if (trsv_stream_supported<T>(lb, strideC, R, upper, lb.perm, work))
    return launch_trsv_stream<T>(M, lb, C, strideC, ldc, R, upper, lb.perm, work, st);
  // few right-hand sides that fit in shared memory: the resident-RHS kernel
  size_t sm_small = sizeof(T) * ((size_t)lb.N * R + (size_t)lb.NB * R) + sizeof(int) * lb.N;
  size_t stage_d = 0;
  const size_t dbytes = sizeof(T) * (size_t)lb.NB * lb.NB;
  if (sm_small + 16 + dbytes <= 112 * 1024) {       // keep two CTAs per SM
    stage_d = (sm_small + 15) / 16 * 16;
    sm_small = stage_d + dbytes;
  }
  if (R <= 25 && sm_small <= 200 * 1024) {
    const int np = lb.nsteps();
#define TS_LAUNCH(UP, RM)                                                                            \
    do {                                                                                             \
      smem_limit(k_trisolve_smem<T, UP, RM, 1>, 200 * 1024);                                         \
      k_trisolve_smem<T, UP, RM, 1><<<lb.batch, 512, sm_small, st>>>(                                \
          M, lb.strideM, lb.N, lb.NB, np, (const T *)(UP ? lb.Uinv : lb.Linv), C, strideC, ldc, R,   \
          lb.ipiv, stage_d);                                                                         \
    } while (0)
    if (upper) {
      if (R == 9) TS_LAUNCH(true, 9); else if (R <= 4) TS_LAUNCH(true, 4);
      else if (R <= 16) TS_LAUNCH(true, 16); else TS_LAUNCH(true, 25);
    } else {
      if (R == 9) TS_LAUNCH(false, 9); else if (R <= 4) TS_LAUNCH(false, 4);
      else if (R <= 16) TS_LAUNCH(false, 16); else TS_LAUNCH(false, 25);
    }
#undef TS_LAUNCH
    return ADGA_LAUNCH_CHECK();
  }
  const int nph = 256 / lb.NB;
  size_t sm = sizeof(T) * ((size_t)nph * lb.NB * RT + (size_t)lb.NB * RT) + sizeof(int) * lb.N;
  if (upper)
    smem_limit(k_trisolve<T, true>, 200 * 1024);
  else
    smem_limit(k_trisolve<T, false>, 200 * 1024);
  if (!upper && !work) return cudaErrorInvalidValue;
  dim3 g(cdiv_u(R, RT), lb.batch);
  if (upper)
    k_trisolve<T, true><<<g, 256, sm, st>>>(M, lb.strideM, lb.N, lb.NB, lb.nsteps(), (const T *)lb.Uinv,
                                            C, strideC, ldc, R, lb.ipiv, work);
  else
    k_trisolve<T, false><<<g, 256, sm, st>>>(M, lb.strideM, lb.N, lb.NB, lb.nsteps(), (const T *)lb.Linv,
                                             C, strideC, ldc, R, lb.ipiv, work);
  return ADGA_LAUNCH_CHECK();
}

template <typename T>
cudaError_t lu_backsolve(const T *M, const LUBatch &lb, T *C, size_t strideC, int ldc, int R,
                         cudaStream_t st) {
  return trisolve<T>(M, lb, C, strideC, ldc, R, true, nullptr, st);
}

// work: batch * ceil(R/16) * N * 16 elements
template <typename T>
cudaError_t lu_fwdsolve_ws(const T *M, const LUBatch &lb, T *V, size_t strideV, int ldv, int R,
                           T *work, cudaStream_t st) {
  return trisolve<T>(M, lb, V, strideV, ldv, R, false, work, st);
}

template cudaError_t lu_factor<z64>(z64 *, const LUBatch &, bool, trail_fn, void *, cudaStream_t, TrailTiming *,
                                    bool);
template cudaError_t lu_step<z64>(z64 *, const LUBatch &, int, bool, trail_fn, void *, cudaStream_t, TrailTiming *,
                                  bool);
template cudaError_t lu_step<z32>(z32 *, const LUBatch &, int, bool, trail_fn, void *, cudaStream_t, TrailTiming *,
                                  bool);
template cudaError_t lu_factor<z32>(z32 *, const LUBatch &, bool, trail_fn, void *, cudaStream_t, TrailTiming *,
                                    bool);
template cudaError_t lu_trail_cuda<z64>(z64 *, const LUBatch &, int, int, cudaStream_t);
template cudaError_t lu_trail_cuda<z32>(z32 *, const LUBatch &, int, int, cudaStream_t);
template cudaError_t lu_backsolve<z64>(const z64 *, const LUBatch &, z64 *, size_t, int, int, cudaStream_t);
template cudaError_t lu_backsolve<z32>(const z32 *, const LUBatch &, z32 *, size_t, int, int, cudaStream_t);
template cudaError_t lu_fwdsolve_ws<z64>(const z64 *, const LUBatch &, z64 *, size_t, int, int, z64 *,
                                         cudaStream_t);
template cudaError_t lu_fwdsolve_ws<z32>(const z32 *, const LUBatch &, z32 *, size_t, int, int, z32 *,
                                         cudaStream_t);
