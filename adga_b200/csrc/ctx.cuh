// Device-side view of one run: sizes plus pointers to the resident
// one-particle data.  Passed by value to the kernels.
#pragma once
#include "common.cuh"
#include "adga.h"

// Transform path of the bubble and the EOM (k_dft.cu): G^ = DFT over k of the G
// table, the fold mesh m of the q points (q = (n/m).a per axis) with each q's
// linear index a on it, twiddle tables e^{2 pi i j/n} of the k and m axes, and
// two scratch arrays of max(nnu_all m^3 nd2^2, iwf m^3 nd2^2, iwf nkp nd2) elements.
struct DftView {
  const z64 *ghat;               // null: the direct k-sum kernels only
  int m[3];
  int min_points;                // batches with fewer points use the direct kernels
  const int *qlin;               // (nqp)
  const double2 *twk[3], *twm[3];
  z64 *a, *b;
};

struct DevCtx {
  int nd, nd2, nkp, nqp, nkp_eom;
  int nkpx, nkpy, nkpz;
  int iwmax, iwf, iwb;           // one-particle box, two-particle half box, bosonic half box
  int N, R;                      // BSE dimension maxdim = nd2*2*iwf; right-hand sides = nd2
  int iwstart, iwstop;           // chi0 nu range
  int nu_lo, nnu;                // G-table covers nu in [nu_lo, nu_lo + nnu)
  double beta, mu;
  const double *iw;              // iw_data, index n + iwmax
  const z64 *hk;                 // hk(i,j,k) at k*nd2 + i + j*nd
  const z64 *siw, *giw;          // (n + iwmax) + i*2*iwmax
  const z64 *dc;                 // dc(s,i) at s + 2*i
  const z64 *u, *ut;             // nd2 x nd2
  const z64 *ndmft;              // nd
  const int *kq;                 // k-q index, 0-based, (nkp, nqp)
  const int *kqe;                // EOM k-q index, 0-based, (nkp_eom, nqp)
  const int *keom;               // EOM k-points (k_data_eom, 1-based), null for the full mesh
  const z64 *vq;                 // V(q) (nd2, nd2, nqp) in read_vq's layout, null without do_vq
  const z64 *nfock;              // n_fock(k, i, j) (nkp, nd, nd), with vq
  const z64 *gtab;               // G(k, nu): [(nu - nu_lo)*nkp + k][nd2], column-major nd x nd
  DftView dft;
};

// correlated-subspace atom (1-based) of every band, 0 for uncorrelated bands
struct VertexAtoms {
  int a[ADGA_MAX_BANDS];
};

// Kernel launchers (host functions), grouped by source file.
// k_onepart.cu
cudaError_t launch_gtable(const DevCtx &c, z64 *gtab, cudaStream_t st);
cudaError_t launch_kq_index(int nkpx, int nkpy, int nkpz, const int *k_sel, int nk_sel,
                            const int *q_data, int nqp, int one_based, int *ind, cudaStream_t st);
cudaError_t launch_local_diag(const DevCtx &c, int iwb, z64 *c0inv, z64 *c0w, z64 *bubloc_tmp,
                              cudaStream_t st);
cudaError_t launch_local_F(const DevCtx &c, const z64 *chi_loc, const z64 *c0inv, z64 *Frow,
                           cudaStream_t st, bool minus_one = true);
cudaError_t launch_gtable_dot(const DevCtx &c, const z64 *dhk, z64 *gdot, cudaStream_t st);
cudaError_t launch_local_gamma(const DevCtx &c, const z64 *Frow, z64 *gam, z64 *opg, cudaStream_t st);
cudaError_t launch_chi_loc_update(const DevCtx &c, const z64 *gam_d, const z64 *gam_m,
                                  const z64 *c0w, const z64 *bubloc_tmp, z64 *chi_loc_d,
                                  z64 *chi_loc_m, z64 *bubble_loc, cudaStream_t st);
cudaError_t launch_eom_static(const DevCtx &c, z64 *sigma_dmft, cudaStream_t st);
cudaError_t launch_eom_dmft(const DevCtx &c, int iwb, const z64 *gam_d, z64 *sigma_dmft,
                            cudaStream_t st);
cudaError_t launch_mirror_sigma(const DevCtx &c, z64 *sigma, int nk, cudaStream_t st);
cudaError_t launch_calc_chi_qw(const DevCtx &c, z64 *chi_qw, const z64 *interm3,
                               const z64 *chi0_sum, cudaStream_t st);

// k_vertex.cu: read_vertex's transform of g4 (one omega) into chi_loc (device buffers)
cudaError_t launch_vertex_g4(const DevCtx &c, int iwb, int vtype, int W, const VertexAtoms &atoms,
                             const z64 *g4d, const z64 *g4m, z64 *chid, z64 *chim, cudaStream_t st);

// k_vertex.cu: read_threeleg's transform into gamma^w (nd2 x N); 1 + gamma^w; read_chi_loc's
// transform into chi_loc (nd2, nd2, 2 iwb + 1) per channel
cudaError_t launch_threeleg(const DevCtx &c, int iwb, int n3iwf, const VertexAtoms &atoms, const z64 *g3d,
                            const z64 *g3m, z64 *gd, z64 *gm, cudaStream_t st);
cudaError_t launch_one_plus_gamma(const DevCtx &c, const z64 *gam, z64 *opg, cudaStream_t st);
cudaError_t launch_chi_loc_ext(const DevCtx &c, int n2iwb, const VertexAtoms &atoms, int extend, const z64 *rd,
                               const z64 *rm, z64 *od, z64 *om, cudaStream_t st);

// k_postloop.cu: add_siw_dmft on sig (in place), then get_sigma_g_loc (sig_loc, gloc; full
// k mesh) and get_ndga (n_dga_k, n_dga); null outputs are skipped
cudaError_t launch_post_loop(const DevCtx &c, const int *keom, z64 *sig, z64 *sig_loc, z64 *gloc,
                             z64 *n_dga_k, z64 *n_dga, cudaStream_t st);

cudaError_t launch_nfock(const DevCtx &c, z64 *nfock, cudaStream_t st);

// k_vq.cu: V(q) (do_vq)
cudaError_t launch_vq_permute(int nd, int nqp, const z64 *raw, z64 *v, cudaStream_t st);
cudaError_t launch_eom_static_vq(const DevCtx &c, const int *qidx, int npts, z64 *sigma_hf, cudaStream_t st);
cudaError_t launch_vq_resid_extra(const DevCtx &c, int npts, const int *qidx, const z64 *X, const z64 *chi0q,
                                  const z64 *opg_d, z64 *extra, cudaStream_t st);

// k_tangent.cu: forward-mode tangents of one batch (FP64 path)
cudaError_t launch_tan_rhs(const DevCtx &c, int npts, int ch, const z64 *XS, const z64 *Frow, const z64 *XD,
                           const z64 *Fdot, const z64 *dB, z64 *out, cudaStream_t st);
cudaError_t launch_gamq_tan(const DevCtx &c, int npts, const z64 *chi0q, const z64 *dchi0q, const z64 *c0inv,
                            const z64 *Frow_d, const z64 *Fdot_d, z64 *dgq, cudaStream_t st);
cudaError_t launch_zadd(size_t n, const z64 *x, z64 *y, cudaStream_t st);

// k_chi0.cu: chi0q[p] (nd2, nd2, nnu_out) for a batch of points at one omega
// (the G(k-q, nu-omega) factor from g2tab, with its transform g2hat, when given:
// tangents); the transform path when c.dft.ghat is set and the batch is large enough
cudaError_t launch_chi0(const DevCtx &c, int iwb, const int *qidx, int npts, z64 *chi0_all,
                        int nnu_all, cudaStream_t st, const z64 *g2tab = nullptr, const z64 *g2hat = nullptr);

// k_dft.cu: transforms (see DftView)
z64 *dft3(const z64 *src, z64 *x, z64 *y, int batch, const int n[3], const double2 *const tw[3], int C,
          double sign, cudaStream_t st, cudaError_t *err);
cudaError_t launch_gtable_dft(const DevCtx &c, const z64 *gtab, z64 *ghat, z64 *scratch, cudaStream_t st);
cudaError_t launch_chi0_dft(const DevCtx &c, int iwb, const int *qidx, int npts, z64 *chi0_all, int nnu_all,
                            const z64 *ghat1, const z64 *ghat2, cudaStream_t st);
cudaError_t launch_eom_dft(const DevCtx &c, int iwb, const int *qidx, int npts, const z64 *mtot, const z64 *ghat,
                           z64 *sigma, cudaStream_t st);
cudaError_t launch_chi0_finish(const DevCtx &c, const z64 *chi0_all, int nnu_all, int npts,
                               const z64 *bubloc_tmp, z64 *chi0q, z64 *bubble_nl, cudaStream_t st);

// k_bse.cu
template <typename T>
cudaError_t launch_bse_build(const DevCtx &c, int npts, const z64 *chi0q, const z64 *c0inv,
                             const z64 *Frow_d, const z64 *Frow_m, const z64 *opg_d,
                             const z64 *opg_m, T *Tmat, size_t strideM, z64 *gammaqd,
                             const int *qidx, cudaStream_t st, const z32 *F32_m = nullptr);
// FP32 copy of an N x N FP64 matrix (the magnetic F~ of the mixed build)
cudaError_t launch_to32(size_t n, const z64 *x, z32 *y, cudaStream_t st);
// X of point p, channel ch at X + p*sp + ch*sc: N x R column-major (ld ldX)
cudaError_t launch_post(const DevCtx &c, int npts, const z64 *X, size_t sp, size_t sc, int ldX,
                        const z64 *opg_d, const z64 *opg_m, const z64 *gam_d, const z64 *gam_m,
                        const z64 *gammaqd, const z64 *chi0q, const z64 *c0w, z64 *chi_qw_d,
                        z64 *chi_qw_m, z64 *mtot, z64 *etad, z64 *etam, const int *qidx, cudaStream_t st);
cudaError_t launch_eom_dynamic(const DevCtx &c, int iwb, const int *qidx, int npts,
                               const z64 *mtot, z64 *sigma_nl, cudaStream_t st);

// k_refine.cu
cudaError_t launch_init_x(const z32 *T32, size_t strideM, int N, int R, int nmat, z64 *X, cudaStream_t st);
// rnorm (nullable): per-matrix max |re| + |im| of the FP64 residual, atomicMax on the bit patterns;
// Bpt (nullable): per-point right-hand sides in X's layout instead of (1+gamma^w) (tangent solves)
// ri8 (k_resid_i8.cu context, or null for the FP64 CUDA-core GEMM): the product
// X D F~ from exact int8 slices on the tensor cores; fgen names the current F~
// (its slices are cut again when it changes)
cudaError_t launch_residual(const DevCtx &c, int npts, const z64 *X, const z64 *chi0q,
                            const z64 *c0inv, const z64 *Frow_d, const z64 *Frow_m,
                            const z64 *opg_d, const z64 *opg_m, z64 *XD, z32 *V, const z64 *extra_d,
                            unsigned long long *rnorm, cudaStream_t st, const z64 *Bpt = nullptr,
                            void *ri8 = nullptr, long long fgen = 0);
// the int8-slice residual (k_resid_i8.cu)
cudaError_t ri8_setup(void **ctx, int N, int R, int cap);
void ri8_free(void *ctx);
int ri8_error(void *ctx);
cudaError_t ri8_residual(void *ctx, const DevCtx &dc, int npts, const z64 *XD, const z64 *X,
                         const z64 *Frow_d, const z64 *Frow_m, long long fgen, const z64 *opg_d,
                         const z64 *opg_m, z32 *V, const z64 *extra_d, unsigned long long *rnorm, const z64 *Bpt,
                         cudaStream_t st);
cudaError_t launch_xd(const DevCtx &c, int npts, const z64 *X, const z64 *chi0q, const z64 *c0inv, z64 *XD,
                      bool minus_one, cudaStream_t st);
cudaError_t launch_update(int per, int nmat, const z32 *V, z64 *X, unsigned long long *norms,
                          const int *active, cudaStream_t st);
