/*
 * adga.h -- C ABI of the B200 ladder hot path (libadga_b200.so).
 *
 * Every entry point replaces one call site or routine of the reference's
 * per-(q, omega) loop (paths relative to the reference project root).  All
 * arrays use the reference's Fortran layouts: column-major, complex values as
 * interleaved (re, im) doubles (adga_z is layout-identical to Fortran
 * complex(kind=8), C99 double _Complex and cuDoubleComplex), frequency axes
 * stored from their lowest index.  Indices that the Fortran code passes
 * 1-based (iq, k-point indices, q_data) stay 1-based here.
 *
 * Return value of every int function: 0 = ok; > 0 = LAPACK-style info (the
 * 1-based index of the first exactly-zero pivot of an LU); < 0 = one of the
 * ADGA_E* codes below.  adga_last_error() gives the message, in the spirit
 * of the reference's (erstr, ierr) pairs (src/lapack_module.f90:40-70).
 *
 * Threading: calls on one handle must not overlap; distinct handles are
 * independent.  Streams and CUDA graphs stay internal to the library.
 */
#ifndef ADGA_B200_H
#define ADGA_B200_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct adga_z { double re, im; } adga_z;

/* error codes (negative returns) */
#define ADGA_EINVAL   (-1)   /* bad argument or inconsistent sizes          */
#define ADGA_ECUDA    (-2)   /* CUDA runtime / driver error                  */
#define ADGA_ENOMEM   (-3)   /* device allocation failed                     */
#define ADGA_ETIMEOUT (-4)   /* a bounded device wait gave up                */
#define ADGA_ESTATE   (-5)   /* call order violated (e.g. vertex not set)    */
#define ADGA_ENOCONV  (-6)   /* mixed-precision refinement did not converge  */

/* precision modes of the BSE solve */
#define ADGA_FP64  0   /* complex FP64 LU + solves (the plain GPU path)            */
#define ADGA_MIXED 1   /* complex FP32 LU, BF16x3 tensor-core updates, FP64 refine */

/*
 * Sizes and scalars of the run.  The reference keeps these as module
 * globals (src/parameters_module.f90:43-58) that every hot routine reads
 * implicitly; here they are passed once.
 */
typedef struct adga_dims {
  int ndim;                    /* orbitals                                   */
  int nkpx, nkpy, nkpz;        /* k-grid (nkp = product)                      */
  int nqpx, nqpy, nqpz;        /* q-volume (nqp = product), q-grid on k-grid  */
  int iwmax;                   /* one-particle box -iwmax..iwmax-1            */
  int iwfmax_small;            /* two-particle box -iwf..iwf-1                */
  int iwbmax_small;            /* bosonic -iwb..iwb                           */
  int iwstart, iwstop;         /* chi0 nu range (src/config_module.f90:467-477)*/
  int do_chi, do_eom;          /* calc-chi / calc-eom                          */
  int nkp_eom;                 /* k points of the EOM (nkp for the full mesh) */
  double beta, mu;
} adga_dims;

typedef struct adga_handle adga_handle;

/*
 * Upload the one-particle data, build G(k, nu) on the device and the k-q
 * lookup tables.  Replaces the set-up of src/main.F90:161-375 that the loop
 * depends on: iw_data (config_init, src/config_module.f90:510-513), hk
 * (read_hk_w2w), siw/giw/dc, u/u_tilde (create_u / read_u), n_dmft
 * (get_ndmft), q_data (generate_q_vol, src/kq_tools.f90:42-57) and
 * k_data_eom.  Shapes (Fortran): iw_data(-iwmax:iwmax-1), hk(ndim,ndim,nkp),
 * siw/giw(-iwmax:iwmax-1,ndim), dc(2,ndim), u/u_tilde(ndim2,ndim2),
 * n_dmft(ndim), q_data(nqp) 1-based k indices, k_data_eom(nkp_eom) 1-based
 * (NULL = 1..nkp).
 */
int adga_create(const adga_dims *d, const double *iw_data, const adga_z *hk,
                const adga_z *siw, const adga_z *giw, const adga_z *dc,
                const adga_z *u, const adga_z *u_tilde, const adga_z *n_dmft,
                const int *q_data, const int *k_data_eom, adga_handle **out);
int adga_destroy(adga_handle *h);
const char *adga_last_error(const adga_handle *h);
int adga_device_bytes(const adga_handle *h, long long *bytes);

/*
 * Stage chi_loc^{dens,magn}(omega = iwb) on the device, as returned by
 * read_vertex (src/hdf5_module.f90:629-773): two maxdim x maxdim complex
 * matrices in the compound index (i1 + nu*ndim2, i2 + nu'*ndim2).  Replaces
 * the per-omega read at src/main.F90:525.  Every omega of a later
 * adga_ladder_run must have been staged.
 */
int adga_set_vertex(adga_handle *h, int iwb, const adga_z *chi_loc_dens,
                    const adga_z *chi_loc_magn);

/* Vertex types of the two-particle input (vertex_type, src/parameters_module.f90:74). */
#define ADGA_VERTEX_FULL_G4      0   /* full two-particle Green's function      */
#define ADGA_VERTEX_CONNECTED_G4 1   /* connected part                          */
#define ADGA_VERTEX_CHI_G4       2   /* generalised susceptibility chi          */
#define ADGA_MAX_BANDS 32

/*
 * Vertex ingest: read_vertex's transform (src/hdf5_module.f90:629-773) on
 * the device.  g4_dens / g4_magn hold the local two-particle Green's
 * function of omega = iwb as w2dynamics stores it and read_vertex places it
 * (before its beta factor, :700,711): Fortran order
 * g4(ndim, ndim, -iwfmax_g4:iwfmax_g4-1, ndim, ndim, -iwfmax_g4:iwfmax_g4-1),
 * iwfmax_g4 >= iwfmax_small.  The library applies the beta factor, the
 * compound index of the small box and the disconnected terms of vertex_type
 * (ADGA_VERTEX_*), and stages the result as adga_set_vertex would.
 * nineq and ndims(nineq, 2) (Fortran order: correlated, then uncorrelated
 * band counts per inequivalent atom) decide which legs share a correlated
 * subspace (index2cor, src/aux.f90:190-221); their band counts must sum to
 * ndim.  Replaces read_vertex's loop at src/hdf5_module.f90:718-770.
 */
int adga_set_vertex_g4(adga_handle *h, int iwb, int vertex_type, int iwfmax_g4, int nineq,
                       const int *ndims, const adga_z *g4_dens, const adga_z *g4_magn);

/* The same transform, returning chi_loc^{dens,magn} (maxdim x maxdim,
 * column-major) to host memory instead of staging it. */
int adga_vertex_transform(adga_handle *h, int iwb, int vertex_type, int iwfmax_g4, int nineq,
                          const int *ndims, const adga_z *g4_dens, const adga_z *g4_magn,
                          adga_z *chi_loc_dens, adga_z *chi_loc_magn);

/*
 * External three-leg vertex (external_threelegs, src/main.F90:560-561):
 * read_threeleg's transform (src/hdf5_module.f90:860-880) on the device.
 * g3_dens / g3_magn: g3(ndim, ndim, ndim, ndim, 2*n3iwf) as w2dynamics stores
 * it for omega = iwb (Matsubara -n3iwf..n3iwf-1, before the beta factor of
 * :829,838), n3iwf >= iwfmax_small.  The resulting gamma^w(ndim2, maxdim)
 * replaces the sum over the F~ rows for that omega (1+gamma^w follows);
 * adga_get_gamma_w returns it.  nineq / ndims as for adga_set_vertex_g4.
 */
int adga_set_threeleg(adga_handle *h, int iwb, int n3iwf, int nineq, const int *ndims,
                      const adga_z *g3_dens, const adga_z *g3_magn);

/*
 * External local susceptibility (external_chi_loc, src/main.F90:407-411):
 * read_chi_loc's transform (src/hdf5_module.f90:958-993) on the device.
 * chi_dens / chi_magn: chi(ndim, ndim, ndim, ndim, 2*n2iwb+1) (bosonic
 * -n2iwb..n2iwb, n2iwb >= iwbmax_small).  From then on the handle's chi_loc
 * outputs are these (the loop no longer builds them from gamma^w, and the
 * local bubble is not added at assembly, src/main.F90:933-936).
 */
int adga_set_chi_loc_ext(adga_handle *h, int n2iwb, int nineq, const int *ndims,
                         const adga_z *chi_dens, const adga_z *chi_magn);

/*
 * Non-local interaction V(q) (do_vq, read_vq at src/main.F90:497-498).
 * vq(ndim, ndim, ndim, ndim, nqp): V(q)_{ijkl} for the handle's q points in
 * q_data order, as read_vq reads it (src/interaction_module.f90:75-104); the
 * library applies read_vq's index map (:107-119), computes n_fock (get_nfock,
 * src/one_particle_quant_module.f90:316-342) and from then on adds the V(q)
 * terms: the density-channel BSE term 2 beta^-2 chi0^q v (1+gamma^w_d)
 * (src/main.F90:710-719, also in the mixed refinement residual), the m_tot
 * terms (src/eom_module.f90:187-205) and calc_eom_static's non-local Hartree
 * and Fock parts into sigma_hf (src/eom_module.f90:70-108).  NULL switches
 * the interaction off.
 */
int adga_set_vq(adga_handle *h, const adga_z *vq);

/* index2component_band (src/aux.f90:169-186): the 1-based band pattern
 * b[0..3] of a 1-based vertex group index ind over nbands bands (the group
 * names of the w2dynamics vertex file).  Host only; returns 0 or ADGA_EINVAL. */
int adga_index2component_band(int nbands, int ind, int *b);

/*
 * Post-loop assembly of the self-energy (src/main.F90:869-890) on the GPU:
 *   add_siw_dmft     (src/eom_module.f90:237-251): sigma_sum(i,i,nu,k) += siw(nu,i);
 *   get_sigma_g_loc  (src/one_particle_quant_module.f90:129-187): the k-summed DGA
 *                    self-energy sigma_loc(ndim,ndim,-iwfmax_small:iwfmax_small-1) and
 *                    Green's function gloc(-iwmax:iwmax-1,ndim,ndim) (DGA Sigma inside
 *                    the vertex box, siw outside, gloc(-nu-1) = gloc(nu)^dagger);
 *                    needs the EOM on the full k mesh;
 *   get_ndga         (src/one_particle_quant_module.f90:344-394): n_dga_k(nkp_eom,ndim,ndim)
 *                    and n_dga(ndim) (complex, zero imaginary part, as declared at
 *                    src/parameters_module.f90:61).
 * sigma_sum (ndim,ndim,-iwfmax_small:iwfmax_small-1,nkp_eom) holds the reduced non-local
 * self-energy (src/main.F90:845-852) on entry and sigma_sum + siw on exit; NULL uses
 * this handle's own accumulated (mirrored) Sigma_nl and leaves it unchanged.  Any
 * output may be NULL to skip it.
 */
int adga_post_loop(adga_handle *h, adga_z *sigma_sum, adga_z *sigma_loc, adga_z *gloc,
                   adga_z *n_dga_k, adga_z *n_dga);

/* Zero the device accumulators (chi, bubble, Sigma) before a run. */
int adga_reset_outputs(adga_handle *h);

/* statistics of the last adga_ladder_run */
typedef struct adga_run_stats {
  int points;                  /* (q, omega) points processed                  */
  int lu_info_nonzero;         /* points whose LU hit an exactly-zero pivot    */
  int mixed_fallbacks;         /* mixed points re-solved in FP64               */
  int max_refine_iters;        /* largest count of FP64 residuals of a batch
                                  (its tangent solves included)                */
  double max_refine_resid;     /* largest final relative correction, or its
                                  bound when the last solve was skipped        */
  double ms_total;             /* device time of the run (CUDA events)         */
  double ms_chi0, ms_bse, ms_lu, ms_post, ms_eom;   /* per-stage device time   */
  long long kernel_launches;   /* kernels this run launched                      */
  double ms_trail;             /* device time of the timed LU trailing updates   */
  double trail_gflop;          /* their algorithmic flops (8 m n k per complex)  */
  int trail_launches;          /* number of timed trailing-update launches       */
  double trail_gbytes;         /* their algorithmic HBM bytes (C r+w, L21, U12)  */
} adga_run_stats;

/*
 * The batched (q, omega) loop of src/main.F90:486-799 over the compound
 * points qwstart..qwstop (1-based, omega outer, q inner: qw(1,i) = iwb,
 * qw(2,i) = iq, src/main.F90:381-389).  Results accumulate in device
 * buffers exactly as the reference's arrays do (read them with
 * adga_get_outputs): chi_qw_dens/magn and bubble_nl per point, bubble_loc,
 * chi_loc_dens/magn per omega (only where the block holds iq = 1, like the
 * reference), sigma_nl (ndim,ndim,-iwf:iwf-1,nkp_eom), sigma_dmft, sigma_hf.
 * precision is ADGA_FP64 or ADGA_MIXED.  status (qwstop-qwstart+1 ints, may
 * be NULL) receives the per-point LU info (> 0 zero pivot) or -1 for a
 * mixed point that fell back to FP64.
 */
int adga_ladder_run(adga_handle *h, int qwstart, int qwstop, int precision,
                    int *status, adga_run_stats *stats);

/*
 * Tunable choices of the ADGA_MIXED path, per handle, and the autotuner that
 * picks them by measurement.  No counterpart in the reference (it has no GPU
 * path); they select kernel variants, never the arithmetic's result beyond
 * the mixed path's tolerance.
 *   factor  0: complex FP32 LU with BF16x3 tensor-core updates and FP64
 *              refinement; 1: the FP64 LU (no refinement), for sizes where
 *              it is the faster way to the same accuracy
 *   pairs   2: tensor-core updates delayed in three-step groups (K = 192
 *              per C pass); 3: four-step groups (K = 256); 1: two-step
 *              groups (K = 128); 0: one update per step (K = 64)
 *   tri_tc  1: the L21 / U12 panel products on the tensor cores, writing the
 *              update operands directly; 0: FP32 CUDA-core tile products and
 *              separate operand-split kernels
 *   batch   points per batch (0: as many as 60% of the free memory holds)
 *   resid   1: the FP64 refinement residual's product X D F~ formed exactly
 *              from int8 slices on the tensor cores; 0: FP64 CUDA-core GEMM
 *   trsv_tc 1: the triangular solves of the FP32 factors on the tensor cores
 *              (3-term TF32 split; N <= 1088, ndim^2 <= 16); 0: streaming
 *              CUDA-core solves
 * A new handle starts at {0, 2, 1, 0, 1, 1} (the environment switches
 * ADGA_NO_PAIRS, ADGA_TRI_TILE, ADGA_BATCH, ADGA_RESID_FP64 and
 * ADGA_TRSV_STREAM override it).
 */
typedef struct adga_tune {
  int factor, pairs, tri_tc, batch, resid, trsv_tc;
} adga_tune;
typedef struct adga_tune_trial {
  adga_tune tune;
  double ms;        /* device time of the sample run (CUDA events)                 */
  double err;       /* max relative difference of chi_d, chi_m, Sigma from FP64    */
  int accepted;     /* err <= tol                                                   */
} adga_tune_trial;
int adga_set_tune(adga_handle *h, const adga_tune *t);
int adga_get_tune(const adga_handle *h, adga_tune *t);
/* Run the candidate configurations of the mixed path on the points
 * qwstart..qwstop (each once to warm up, once timed), compare chi_qw_dens,
 * chi_qw_magn and sigma_nl with the FP64 path on the same points, and keep on
 * the handle the fastest configuration within tol (<= 0: 1e-8).  trials
 * (room for max_trials, may be NULL) receives every measurement, *ntrials
 * their count, *best the choice.  The accumulators are reset afterwards. */
int adga_autotune(adga_handle *h, int qwstart, int qwstop, double tol, adga_tune_trial *trials,
                  int max_trials, int *ntrials, adga_tune *best);

/* Host copies of the accumulators; any pointer may be NULL. */
typedef struct adga_outputs {
  adga_z *chi_qw_dens;     /* (ndim2, ndim2, qwstart:qwstop) of the last run   */
  adga_z *chi_qw_magn;
  adga_z *bubble_nl;
  adga_z *bubble_loc;      /* (ndim2, ndim2, -iwb:iwb)                          */
  adga_z *chi_loc_dens;
  adga_z *chi_loc_magn;
  adga_z *sigma_nl;        /* (ndim, ndim, -iwf:iwf-1, nkp_eom), mirrored       */
  adga_z *sigma_dmft;      /* (ndim, ndim, -iwf:iwf-1)                          */
  adga_z *sigma_hf;        /* (ndim, ndim, nkp_eom)                             */
} adga_outputs;
int adga_get_outputs(adga_handle *h, const adga_outputs *o);

/*
 * Derivatives of the FP64 ladder outputs along up to ADGA_MAX_TANGENTS
 * parameter directions at once (forward-mode tangents; the gradient of any
 * scalar of chi and Sigma follows by contraction).  Direction dir is given by
 * its input tangents, each optional (NULL = zero): dH(k) (ndim, ndim, nkp), du
 * and du_tilde (ndim2, ndim2), and per omega dchi_loc^{dens,magn}
 * (maxdim x maxdim).  The DMFT one-particle inputs (siw, giw, mu, dc,
 * n_dmft) are held fixed.  The tangent follows every stage of the loop:
 * dG = G dH G in chi0 and the EOM, d(F~) = sym(dchi_loc) chi0_loc^-1,
 * dX = (d(1+gamma^w) - X dA) A^-1 through the BSE (d(A^-1) = -A^-1 dA A^-1,
 * with the LU factors of the forward solve), the chi sums and m_tot.
 * adga_ladder_run_tangent runs the ladder over qwstart..qwstop once in the
 * given precision (its forward outputs accumulate as with adga_ladder_run)
 * together with every direction set: ADGA_FP64 solves the tangents with the
 * FP64 LU factors, ADGA_MIXED with the FP32 factors and FP64 refinement
 * (ADGA_ENOCONV if a tangent's refinement does not converge);
 * adga_get_tangent_outputs returns direction dir in the layouts of
 * adga_get_outputs (bubble_loc and sigma_hf: zero).  Not with V(q).
 * adga_clear_tangents drops every direction.
 */
#define ADGA_MAX_TANGENTS 4
int adga_set_tangent(adga_handle *h, int dir, const adga_z *dhk, const adga_z *du,
                     const adga_z *du_tilde);
int adga_set_vertex_tangent(adga_handle *h, int dir, int iwb, const adga_z *dchi_loc_dens,
                            const adga_z *dchi_loc_magn);
int adga_ladder_run_tangent(adga_handle *h, int qwstart, int qwstop, int precision, int *status,
                            adga_run_stats *stats);
int adga_get_tangent_outputs(adga_handle *h, int dir, const adga_outputs *o);
int adga_clear_tangents(adga_handle *h);


/* ---- per-routine entry points (one (q, omega) point, host buffers) ---- */

/* diag of chi0_loc / chi0_loc^-1 at (iwf, iwb) as ndim2 x ndim2 matrices;
 * get_chi0_loc / get_chi0_loc_inv (src/one_particle_quant_module.f90:192-225) */
int adga_get_chi0_loc(adga_handle *h, int iwf, int iwb, adga_z *chi0_loc);
int adga_get_chi0_loc_inv(adga_handle *h, int iwf, int iwb, adga_z *chi0_loc_inv);

/* k-summed bubble chi0q(ndim2,ndim2,-iwf:iwf-1) at (iq, iwb) and the
 * bubble_nl update of src/main.F90:644-663 (bubble_nl may be NULL; it is
 * overwritten with sum_nu chi0 / beta^2 - bubble_loc(iwb)).  Replaces the
 * accumulate_chi0 k-loop (src/one_particle_quant_module.f90:228-290). */
int adga_chi0_q(adga_handle *h, int iq, int iwb, adga_z *chi0q, adga_z *bubble_nl);

/* BSE build + both inversions + eta for one point, src/main.F90:674-757.
 * Needs adga_set_vertex(iwb).  Outputs (ndim2, maxdim): etaqd, etaqm,
 * gammaqd (any may be NULL). */
int adga_bse_point(adga_handle *h, int iq, int iwb, int precision,
                   adga_z *etaqd, adga_z *etaqm, adga_z *gammaqd, int *lu_info);

/* local gamma^w_d/m (ndim2, maxdim) of omega = iwb (src/main.F90:557-571) */
int adga_get_gamma_w(adga_handle *h, int iwb, adga_z *gammawd, adga_z *gammawm);

/* chi_qw += beta^-2 sum_{nu,i3} interm3(:,{i3,nu}) chi0_sum(i3,:,nu);
 * calc_chi_qw (src/susc_module.f90:34-56) */
int adga_calc_chi_qw(adga_handle *h, adga_z *chi_qw, const adga_z *interm3,
                     const adga_z *chi0_sum);

/* calc_eom_dynamic (src/eom_module.f90:165-233), V(q) = 0:
 * sigma_nl(ndim,ndim,-iwf:iwf-1,nkp_eom) is accumulated in place. */
int adga_calc_eom_dynamic(adga_handle *h, const adga_z *etaqd, const adga_z *etaqm,
                          const adga_z *gammaqd, int iwb, int iq, adga_z *sigma_nl);

/* calc_eom_dmft (src/eom_module.f90:115-161) and the local Hartree term of
 * calc_eom_static (src/eom_module.f90:52-70); sigma_dmft(ndim,ndim,-iwf:iwf-1)
 * is accumulated in place. */
int adga_calc_eom_dmft(adga_handle *h, const adga_z *gammawd, int iwb, adga_z *sigma_dmft);
int adga_calc_eom_static(adga_handle *h, int iq, adga_z *sigma_dmft);

/* In-place inverse of an n x n complex matrix (lda = n) on the GPU:
 * drop-in for inverse_matrix_z (src/lapack_module.f90:40-70).  ierr gets the
 * LAPACK-style info, erstr (>= 200 chars, may be NULL) the reference's
 * message ("ERROR in ZGETRF") on failure. */
int adga_inverse_matrix_z(adga_z *M, int n, int *ierr, char *erstr);

/* Inverse of an n x n complex matrix held in device memory, allocating no
 * device memory: for callers that cannot call cudaMalloc (their device
 * memory belongs to another allocator, or the library must not grow the
 * footprint).  M_dev (n x n, column-major) is read, Minv_dev receives the
 * inverse; both are device pointers owned by the caller.  All scratch sits in
 * one file-scope device array of ADGA_NOALLOC_MAX_N-sized buffers (about
 * 2.6 MB per GPU, held until exit); n > ADGA_NOALLOC_MAX_N returns
 * ADGA_EINVAL.  The first call on a device looks up that array's address
 * (cudaGetSymbolAddress): make it before any stream capture.  Calls share
 * the array, so calls that overlap on the GPU race.  stream may be NULL (the
 * default stream); the call waits for the stream and returns the LAPACK-style
 * info (> 0: exactly zero pivot, the inverse is then not usable), also stored
 * in *ierr when ierr is non-NULL.  No counterpart in the reference. */
#define ADGA_NOALLOC_MAX_N 256
int adga_inverse_matrix_z_noalloc(const adga_z *M_dev, adga_z *Minv_dev, int n, int *ierr,
                                  void *stream);

/* k - q index table ind(nkp_sel, nqp) (1-based), index_kq / index_kq_eom
 * (src/kq_tools.f90:59-108); k_sel NULL = all k. */
int adga_index_kq(int nkpx, int nkpy, int nkpz, const int *q_data, int nqp,
                  const int *k_sel, int nk_sel, int *ind);

/* q-volume q_data(nqp), generate_q_vol (src/kq_tools.f90:42-57). */
int adga_generate_q_vol(int nkpx, int nkpy, int nkpz, int nqpx, int nqpy,
                        int nqpz, int *q_data);

/* Kanamori U for one atom of ndim correlated bands (interaction_mode 1):
 * u({k,i},{j,l}) = U_ijkl, u_tilde({k,i},{j,l}) = U_ijlk;
 * create_u (src/interaction_module.f90:182-291). Umat (ndim^4, may be NULL). */
int adga_create_u(int ndim, double Udd, double Vdd, double Jdd, double *Umat,
                  adga_z *u, adga_z *u_tilde);

#ifdef __cplusplus
}
#endif
#endif /* ADGA_B200_H */
