// Batched complex LU with partial pivoting and blocked triangular solves.
//
// Replaces the zgetrf/zgetri pair of inverse_matrix_z (src/lapack_module.f90:40-70)
// on the BSE matrices of src/main.F90:734-737.  The matrices are the
// transposed BSE matrices T = A^T with the right-hand sides (1+gamma^w)^T
// appended as extra columns, so that one factorisation P T = L U also
// produces L^-1 P B^T, and X = B A^-1 follows from one back substitution
// with U (the reference forms the full inverse instead).
//
// Layout: matrix b at base + b*strideM, column-major, ld = N rows,
// ncols = N + R columns.  ipiv[b*N + i] holds the 0-based row swapped with
// row i (LAPACK convention), info[b] the 1-based index of the first exactly
// zero pivot.  Linv / Uinv hold the inverses of the NB x NB diagonal blocks
// (ld NB) per matrix and step: they turn every triangular solve into small
// GEMMs.
#pragma once
#include "common.cuh"

// Row-interchange map of one step, per matrix: [count, dst0, src0, dst1, src1, ...]
// (after the step's interchanges row dst holds what row src held before).
constexpr int RMAP_STRIDE = 520;   // >= 1 + 2 * (2 * 128) entries

struct LUBatch {
  int N, ncols, batch, NB;
  size_t strideM;
  int *ipiv, *info;
  void *Linv, *Uinv;        // [batch][nsteps][NB*NB] of the element type
  int *rmap;                // [batch][RMAP_STRIDE]
  int *perm = nullptr;      // [batch][N] row i of P B = row perm[i] of B (lu_build_perm); optional
  bool nopiv = false;       // factored without row interchanges (P = 1)
  int *tc_err = nullptr;    // FP32 solves on the tensor cores (k_trsv_tc.cu) where they apply:
                            // the device flag their bounded waits report to; null: streaming solves
  int nsteps() const { return (N + NB - 1) / NB; }
};

// Trailing update C -= A B of one step (rows r0.., cols c0..), pluggable so
// that the mixed path can route it to the tensor cores.  ev0 / ev1 (may be
// null) are recorded around the GEMM launch itself, operand staging excluded.
typedef cudaError_t (*trail_fn)(void *ctx, int J, int jb, cudaStream_t st, cudaEvent_t ev0, cudaEvent_t ev1);

// Optional timing of the trailing updates: events[2*s], events[2*s+1]
// bracket the update of step s (pass nullptr to skip).
struct TrailTiming {
  cudaEvent_t *ev = nullptr;   // 2 * nsteps events, created by the caller
  int n = 0;                   // number of pairs recorded
  double gflop = 0.0;          // algorithmic flops of the recorded updates
  double gbytes = 0.0;         // algorithmic HBM bytes: C read+write, L21 and U12 read once
};
// nopiv: no row interchanges (identity ipiv, empty maps); the mixed path's
// FP32 factorisation, whose refinement falls back to the pivoted FP64 path
template <typename T>
cudaError_t lu_factor(T *M, const LUBatch &lb, bool apply_left, trail_fn trail, void *trail_ctx,
                      cudaStream_t st, TrailTiming *tt = nullptr, bool nopiv = false);
// one step s (panel, block inverses, interchanges + U12, trailing update)
template <typename T>
cudaError_t lu_step(T *M, const LUBatch &lb, int s, bool apply_left, trail_fn trail, void *trail_ctx,
                    cudaStream_t st, TrailTiming *tt = nullptr, bool nopiv = false);
// Delayed updates of the unpivoted FP32 factorisation (tensor cores) in groups of G
// steps (G = 2 or 3): after step g of a group (steps Js[i], widths jbs[i], i <= g),
// `update` applies the group's updates so far to what step g + 1 reads (wide = false)
// or, after the group's last step, to the rest (wide = true).
// tri (optional): L21 and U12 of step (J, jb) in place of the CUDA-core tile
// products, also writing operand staging set `set` (the step's index in its group)
struct GroupOps {
  cudaError_t (*update)(void *ctx, int nst, const int *Js, const int *jbs, bool wide, cudaStream_t st,
                        cudaEvent_t ev0, cudaEvent_t ev1);
  void *ctx;
  cudaError_t (*tri)(void *ctx, int J, int jb, int set, cudaStream_t st) = nullptr;
  int G = 2;
};
cudaError_t lu_factor_groups(z32 *M, const LUBatch &lb, const GroupOps &ops, cudaStream_t st,
                             TrailTiming *tt = nullptr);
// the matrices [first, first + count) of a batch as a batch of their own
template <typename T>
inline LUBatch lu_sub(const LUBatch &lb, int first, int count) {
  LUBatch r = lb;
  const size_t blk = (size_t)lb.nsteps() * lb.NB * lb.NB;
  r.batch = count;
  r.ipiv = lb.ipiv + (size_t)first * lb.N;
  r.info = lb.info + first;
  r.Linv = (T *)lb.Linv + (size_t)first * blk;
  r.Uinv = (T *)lb.Uinv + (size_t)first * blk;
  r.rmap = lb.rmap + (size_t)first * RMAP_STRIDE;
  r.perm = lb.perm ? lb.perm + (size_t)first * lb.N : nullptr;
  return r;
}
template <typename T>
cudaError_t lu_trail_cuda(T *M, const LUBatch &lb, int J, int jb, cudaStream_t st);
// U Y = C in place (C: N x R columns at C + b*strideC, ld ldc)
template <typename T>
cudaError_t lu_backsolve(const T *M, const LUBatch &lb, T *C, size_t strideC, int ldc, int R,
                         cudaStream_t st);
// z = L^-1 P r in place (r: N x R columns at V + b*strideV, ld ldv); needs the
// interchanges applied to the left columns too (apply_left in lu_factor).
// work: batch * ceil(R/16) * N * 16 elements.
template <typename T>
cudaError_t lu_fwdsolve_ws(const T *M, const LUBatch &lb, T *V, size_t strideV, int ldv, int R,
                           T *work, cudaStream_t st);
// the factorization's row permutation, from ipiv, into perm[batch][N]
cudaError_t lu_build_perm(const LUBatch &lb, int *perm, cudaStream_t st);
// streaming solves (k_trsv.cu): NB = 64, R <= 25; the forward one needs lb.perm and work
template <typename T>
bool trsv_stream_supported(const LUBatch &lb, size_t strideC, int R, bool upper, const int *perm,
                           const T *work);
// tensor-core solves of FP32 factors (k_trsv_tc.cu): NB = 64, R <= 16, N <= 1088 and even,
// the forward one only without row interchanges; needs lb.tc_err
bool trsv_tc_supported(const LUBatch &lb, int R, bool upper);
cudaError_t launch_trsv_tc(const z32 *M, const LUBatch &lb, z32 *C, size_t strideC, int ldc, int R, bool upper,
                           cudaStream_t st);
template <typename T>
cudaError_t launch_trsv_stream(const T *M, const LUBatch &lb, T *C, size_t strideC, int ldc, int R,
                               bool upper, const int *perm, T *work, cudaStream_t st);
