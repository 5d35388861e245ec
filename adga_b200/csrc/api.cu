// C ABI of libadga_b200: handle, data staging and the batched (q, omega)
// loop of src/main.F90:486-799 on one GPU.  See include/adga.h for the
// contract of every entry point.
#include "adga.h"
#include "ctx.cuh"
#include "lu.cuh"
#define GINV_MAXND_HOST 8   // ndim limit of the small inverses (ginv.cuh)
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

// tensor-core trailing update of the mixed path (k_tc.cu)
cudaError_t tc_trail_setup(void **ctx, z32 *M, const LUBatch &lb, cudaStream_t st);
cudaError_t tc_trail_run_range(void *ctx, int first, int count, int J, int jb, cudaStream_t st,
                               cudaEvent_t ev0, cudaEvent_t ev1);

// a matrix range of the tensor-core trailing-update context; staged: the step
// kernels (tc_tri_step) write the operand staging, the updates only run the GEMMs
struct TcRange { void *ctx; int first, count; bool staged = false; };
static cudaError_t tc_trail_range_fn(void *r, int J, int jb, cudaStream_t st, cudaEvent_t ev0,
                                     cudaEvent_t ev1) {
  TcRange *x = (TcRange *)r;
  return tc_trail_run_range(x->ctx, x->first, x->count, J, jb, st, ev0, ev1);
}
void tc_trail_free(void *ctx);
int tc_available();
int tc_trail_error(void *ctx);
int *tc_err_flag(void *ctx);
int tc_pair_supported(void *ctx);
cudaError_t tc_group_update(void *ctx, int first, int count, int nst, const int *Js, const int *jbs, bool wide,
                            cudaStream_t st, cudaEvent_t ev0, cudaEvent_t ev1, bool staged);
cudaError_t tc_tri_step(void *ctx, int first, int count, int J, int jb, int set, cudaStream_t st);
static cudaError_t tc_group_fn(void *r, int nst, const int *Js, const int *jbs, bool wide, cudaStream_t st,
                               cudaEvent_t ev0, cudaEvent_t ev1) {
  TcRange *x = (TcRange *)r;
  return tc_group_update(x->ctx, x->first, x->count, nst, Js, jbs, wide, st, ev0, ev1, x->staged);
}
static cudaError_t tc_tri_fn(void *r, int J, int jb, int set, cudaStream_t st) {
  TcRange *x = (TcRange *)r;
  return tc_tri_step(x->ctx, x->first, x->count, J, jb, set, st);
}

// Refinement stop on an estimate: the next correction d = r A^-1 is taken as at
// most kEstSafety * rho * max|r| (rho from the first sweep)
constexpr double kEstSafety = 10.0;

struct TanState;
struct TanWork;

struct adga_handle {
  adga_dims d{};
  DevCtx c{};
  int nw = 0, nnu_all = 0, nd4 = 0;
  bool bigbox = false;
  cudaStream_t st = nullptr, st2 = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr, fork = nullptr, join = nullptr;
  std::string err;
  std::vector<void *> owned;
  // vertex store, one pair per omega
  std::vector<z64 *> vd, vm;
  z64 *g4buf = nullptr;        // staging of the raw vertex / three-leg / chi_loc inputs
  size_t g4cap = 0;
  std::vector<z64 *> tl_d, tl_m;   // external three-leg gamma^w per omega (nd2 x N), or null
  z64 *ext_cld = nullptr, *ext_clm = nullptr;   // external chi_loc (nd2, nd2, nw), or null
  z64 *vq_d = nullptr, *nfock_d = nullptr;       // V(q) and n_fock (do_vq), or null
  z64 *vq_extra = nullptr;                        // density-channel V(q) residual term (mixed)
  TanState *tan[ADGA_MAX_TANGENTS] = {};         // tangent directions, or null
  TanWork *tw = nullptr;                          // their shared work
  bool tan_on = false;                            // inside adga_ladder_run_tangent
  size_t vq_extra_cap = 0;
  // local block
  int diag_iwb = INT_MIN, loc_iwb = INT_MIN;
  z64 *c0inv = nullptr, *c0w = nullptr, *bubtmp = nullptr;
  z64 *Frow_d = nullptr, *Frow_m = nullptr, *gam_d = nullptr, *gam_m = nullptr;
  z64 *opg_d = nullptr, *opg_m = nullptr;
  z32 *Frow32_m = nullptr;       // FP32 copy of F~_m for the mixed build, valid for omega f32_iwb
  int f32_iwb = INT_MIN;
  // accumulators
  z64 *bubble_loc = nullptr, *chi_loc_d = nullptr, *chi_loc_m = nullptr;
  z64 *sigma_nl = nullptr, *sigma_dmft = nullptr, *sigma_hf = nullptr;
  z64 *chi_qw_d = nullptr, *chi_qw_m = nullptr, *bubble_nl = nullptr;
  int out_cap = 0, last_npts = 0;
  // first per-point output slot past the run's points: the FP64 re-solve of
  // mixed points that did not converge writes there, then moves them to their slots
  int fb_base = 0;
  // batch work buffers (sized on demand)
  int cap = 0, cap_prec = -1;
  std::vector<void *> work;
  z64 *chi0_all = nullptr, *chi0q_big = nullptr, *gq = nullptr, *mtot = nullptr;
  z64 *etad = nullptr, *etam = nullptr;
  int *qidx_d = nullptr, *qidx_h = nullptr;
  void *Tm = nullptr, *Linv = nullptr, *Uinv = nullptr;
  int *ipiv = nullptr, *info = nullptr, *rmap = nullptr, *perm = nullptr;
  int NB = 64;
  z64 *X64 = nullptr, *XD = nullptr;
  z32 *V32 = nullptr, *work32 = nullptr;
  unsigned long long *norms = nullptr;
  void *tc = nullptr;
  // refinement settings
  int max_iter = 8;
  bool refine_estimate = true;   // stop on the bounded next correction (ADGA_REFINE_EXACT=1: on a solved one)
  bool mixed_nopiv = true;   // FP32 factorisation without row interchanges (ADGA_MIXED_PIVOT=1: with)
  double tol = 1e-10;   // stop when max|dX| <= tol * max|X| (the error is then far below)
  adga_tune tune{0, 2, 1, 0, 1, 1};   // mixed-path kernel choices (adga_set_tune / adga_autotune)
  void *ri8 = nullptr;            // int8-slice residual context (k_resid_i8.cu), with the mixed work
  long long frow_gen = 0;         // bumped whenever F~ is recomputed (its residual slices go stale)
  // last-run statistics
  adga_run_stats stats{};
};

// one tangent direction
struct TanState {
  bool has_dhk = false;
  z64 *gdot = nullptr, *du = nullptr, *dut = nullptr;
  z64 *ghat_dot = nullptr;                 // transform of gdot (transform path only)
  std::vector<z64 *> vd, vm;               // dchi_loc per omega (N x N), or null
  z64 *Fd = nullptr, *Fm = nullptr, *gd = nullptr, *gm = nullptr;
  int loc_iwb = INT_MIN;
  bool loc_has = false;
  // accumulators
  z64 *chi_loc_d = nullptr, *chi_loc_m = nullptr, *sigma_nl = nullptr, *sigma_dmft = nullptr;
  z64 *chi_qw_d = nullptr, *chi_qw_m = nullptr, *bub_nl = nullptr;
  int out_cap = 0;
  std::vector<void *> owned;
};
// batch work and constants shared by the directions (they run one after another)
struct TanWork {
  z64 *zero_nd4 = nullptr, *zero_N = nullptr, *zero_gam = nullptr, *opg_scr = nullptr, *bub_scr = nullptr;
  std::vector<void *> owned, work;
  int cap = 0;
  z64 *chi0_all = nullptr, *chi0_tmp = nullptr, *chi0q_big = nullptr, *zero_chi0 = nullptr;
  z64 *Xc = nullptr, *XS = nullptr, *XD = nullptr, *Rt = nullptr, *wk = nullptr, *gq = nullptr;
  z64 *cA_d = nullptr, *cA_m = nullptr, *cB_d = nullptr, *cB_m = nullptr, *mA = nullptr, *mB = nullptr;
  z64 *eta_d = nullptr, *eta_m = nullptr;
  int *perm = nullptr;
};
static void tan_free(adga_handle *h);

#define CK(call)                                                                  \
  do {                                                                            \
    cudaError_t _e = (call);                                                      \
    if (_e != cudaSuccess) {                                                      \
      h->err = std::string(#call) + ": " + cudaGetErrorString(_e);                \
      return ADGA_ECUDA;                                                          \
    }                                                                             \
  } while (0)

static int fail(adga_handle *h, int code, const std::string &msg) {
  if (h) h->err = msg;
  return code;
}

static void *dalloc(adga_handle *h, size_t bytes, std::vector<void *> &list) {
  void *p = nullptr;
  if (bytes == 0) bytes = 16;
  if (cudaMalloc(&p, bytes) != cudaSuccess) return nullptr;
  list.push_back(p);
  return p;
}

template <typename P>
static bool alloc_into(adga_handle *h, P *&ptr, size_t count, std::vector<void *> &list) {
  ptr = (P *)dalloc(h, count * sizeof(P), list);
  return ptr != nullptr;
}

static void free_list(std::vector<void *> &list) {
  for (void *p : list) cudaFree(p);
  list.clear();
}

cudaError_t smem_limit_once(const void *kernel, int bytes) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  static std::mutex mu;
  static std::map<std::pair<const void *, int>, int> done;   // (kernel, device) -> limit set
  std::lock_guard<std::mutex> lk(mu);
  auto it = done.find({kernel, dev});
  if (it != done.end() && it->second >= bytes) return cudaSuccess;
  e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess) done[{kernel, dev}] = bytes;
  return e;
}

extern "C" const char *adga_last_error(const adga_handle *h) {
  return h ? h->err.c_str() : "null handle";
}

// ---------------------------------------------------------------------------
// Transform path (k_dft.cu): the fold mesh of the q points, their indices on it,
// twiddles, G^ and scratch.  ADGA_DFT_MIN_POINTS sets the smallest batch that
// uses it (default 4); ADGA_BUBBLE=direct keeps the direct kernels only.  If its
// buffers cannot be allocated the direct kernels are used.
static int gcd_int(int a, int b) {
  while (b) { const int t = a % b; a = b; b = t; }
  return a;
}

static int setup_dft(adga_handle *h, const int *q_data) {
  DevCtx &c = h->c;
  c.dft = DftView{};
  const char *mode = getenv("ADGA_BUBBLE");
  if (mode && !strcmp(mode, "direct")) return 0;
  const char *mp = getenv("ADGA_DFT_MIN_POINTS");
  c.dft.min_points = mp ? std::max(1, atoi(mp)) : 4;
  const int nk[3] = {c.nkpx, c.nkpy, c.nkpz};
  std::vector<int> qc(3 * (size_t)c.nqp);
  int s[3] = {nk[0], nk[1], nk[2]};
  for (int q = 0; q < c.nqp; ++q) {
    const int k0 = q_data[q] - 1;
    if (k0 < 0 || k0 >= c.nkp) return fail(h, ADGA_EINVAL, "q_data outside the k mesh");
    qc[3 * q] = k0 / (nk[1] * nk[2]);
    qc[3 * q + 1] = (k0 / nk[2]) % nk[1];
    qc[3 * q + 2] = k0 % nk[2];
    for (int ax = 0; ax < 3; ++ax) s[ax] = gcd_int(s[ax], qc[3 * q + ax]);
  }
  for (int ax = 0; ax < 3; ++ax) c.dft.m[ax] = nk[ax] / s[ax];
  const int m3 = c.dft.m[0] * c.dft.m[1] * c.dft.m[2];
  std::vector<int> ql(c.nqp);
  for (int q = 0; q < c.nqp; ++q) {
    const int ax = qc[3 * q] / s[0], ay = qc[3 * q + 1] / s[1], az = qc[3 * q + 2] / s[2];
    ql[q] = az + c.dft.m[2] * (ay + c.dft.m[1] * ax);
  }
  std::vector<double2> tw;
  int off[6];
  const int lens[6] = {nk[0], nk[1], nk[2], c.dft.m[0], c.dft.m[1], c.dft.m[2]};
  for (int i = 0; i < 6; ++i) {
    off[i] = (int)tw.size();
    for (int j = 0; j < lens[i]; ++j) {
      const long double ang = 2.0L * 3.141592653589793238462643383279502884L * j / lens[i];
      tw.push_back(make_double2((double)cosl(ang), (double)sinl(ang)));
    }
  }
  const size_t nd4 = (size_t)c.nd2 * c.nd2;
  const size_t scr = std::max({(size_t)h->nnu_all * m3 * nd4, (size_t)c.iwf * m3 * nd4,
                               (size_t)c.iwf * c.nkp * c.nd2, (size_t)c.nnu * c.nkp * c.nd2});
  auto &L = h->owned;
  z64 *ghat, *a, *b;
  int *qlin;
  double2 *twd;
  if (!alloc_into(h, ghat, (size_t)c.nnu * c.nkp * c.nd2, L) || !alloc_into(h, a, scr, L) ||
      !alloc_into(h, b, scr, L) || !alloc_into(h, qlin, c.nqp, L) || !alloc_into(h, twd, tw.size(), L)) {
    h->err.clear();
    c.dft = DftView{};
    return 0;
  }
  CK(cudaMemcpyAsync(qlin, ql.data(), sizeof(int) * c.nqp, cudaMemcpyHostToDevice, h->st));
  CK(cudaMemcpyAsync(twd, tw.data(), sizeof(double2) * tw.size(), cudaMemcpyHostToDevice, h->st));
  c.dft.qlin = qlin;
  for (int i = 0; i < 3; ++i) {
    c.dft.twk[i] = twd + off[i];
    c.dft.twm[i] = twd + off[3 + i];
  }
  c.dft.a = a;
  c.dft.b = b;
  CK(launch_gtable_dft(c, c.gtab, ghat, a, h->st));
  CK(cudaStreamSynchronize(h->st));   // the host vectors above go out of scope
  c.dft.ghat = ghat;
  return 0;
}

extern "C" int adga_create(const adga_dims *d, const double *iw_data, const adga_z *hk,
                           const adga_z *siw, const adga_z *giw, const adga_z *dc,
                           const adga_z *u, const adga_z *u_tilde, const adga_z *n_dmft,
                           const int *q_data, const int *k_data_eom, adga_handle **out) {
  if (!d || !out || !iw_data || !hk || !siw || !giw || !u || !u_tilde || !n_dmft || !q_data)
    return ADGA_EINVAL;
  *out = nullptr;
  if (d->ndim < 1 || d->ndim > 5) return ADGA_EINVAL;
  if (d->nkpx < 1 || d->nkpy < 1 || d->nkpz < 1 || d->nqpx < 1 || d->nqpy < 1 || d->nqpz < 1)
    return ADGA_EINVAL;
  if (d->nkpx % d->nqpx || d->nkpy % d->nqpy || d->nkpz % d->nqpz) return ADGA_EINVAL;
  if (d->iwfmax_small < 1 || d->iwbmax_small < 0) return ADGA_EINVAL;
  if (d->iwmax < d->iwfmax_small + d->iwbmax_small) return ADGA_EINVAL;   // check_freq_range
  if (d->iwstart > -d->iwfmax_small || d->iwstop < d->iwfmax_small - 1) return ADGA_EINVAL;
  if (d->iwstart - d->iwbmax_small < -d->iwmax || d->iwstop + d->iwbmax_small > d->iwmax - 1)
    return ADGA_EINVAL;
  adga_handle *h = new adga_handle();
  h->d = *d;
  DevCtx &c = h->c;
  c.nd = d->ndim; c.nd2 = d->ndim * d->ndim;
  c.nkpx = d->nkpx; c.nkpy = d->nkpy; c.nkpz = d->nkpz;
  c.nkp = d->nkpx * d->nkpy * d->nkpz;
  c.nqp = d->nqpx * d->nqpy * d->nqpz;
  c.nkp_eom = d->nkp_eom > 0 ? d->nkp_eom : c.nkp;
  c.iwmax = d->iwmax; c.iwf = d->iwfmax_small; c.iwb = d->iwbmax_small;
  c.N = c.nd2 * 2 * c.iwf; c.R = c.nd2;
  c.iwstart = d->iwstart; c.iwstop = d->iwstop;
  c.nu_lo = d->iwstart - d->iwbmax_small;
  c.nnu = (d->iwstop + d->iwbmax_small) - c.nu_lo + 1;
  c.beta = d->beta; c.mu = d->mu;
  h->nw = 2 * c.iwb + 1;
  h->nnu_all = d->iwstop - d->iwstart + 1;
  h->bigbox = h->nnu_all != 2 * c.iwf;
  h->nd4 = c.nd2 * c.nd2;
  if (const char *mpv = getenv("ADGA_MIXED_PIVOT")) h->mixed_nopiv = atoi(mpv) == 0;
  if (const char *mr = getenv("ADGA_MAX_REFINE")) h->max_iter = std::max(1, atoi(mr));
  if (const char *re = getenv("ADGA_REFINE_EXACT")) h->refine_estimate = atoi(re) == 0;
  if (getenv("ADGA_NO_PAIRS")) h->tune.pairs = 0;
  if (getenv("ADGA_TRI_TILE")) h->tune.tri_tc = 0;
  if (getenv("ADGA_RESID_FP64")) h->tune.resid = 0;
  if (getenv("ADGA_TRSV_STREAM")) h->tune.trsv_tc = 0;
  const char *ev = getenv("ADGA_NB");
  if (ev) h->NB = std::max(16, std::min(64, atoi(ev) / 8 * 8));   // the LU kernels assume NB <= 64
  if (cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking) != cudaSuccess) {
    delete h;
    return ADGA_ECUDA;
  }
  cudaEventCreate(&h->e0);
  cudaEventCreate(&h->e1);
  cudaEventCreateWithFlags(&h->fork, cudaEventDisableTiming);
  cudaEventCreateWithFlags(&h->join, cudaEventDisableTiming);
  if (cudaStreamCreateWithFlags(&h->st2, cudaStreamNonBlocking) != cudaSuccess) h->st2 = nullptr;
  auto &L = h->owned;
  const int nd = c.nd, nd2 = c.nd2, n2w = 2 * c.iwmax;
  double *iw; z64 *hk_d, *siw_d, *giw_d, *dc_d, *u_d, *ut_d, *nd_d, *gt;
  int *qd, *kq, *kqe, *kde = nullptr;
  bool ok = alloc_into(h, iw, n2w, L) && alloc_into(h, hk_d, (size_t)c.nkp * nd2, L) &&
            alloc_into(h, siw_d, (size_t)n2w * nd, L) && alloc_into(h, giw_d, (size_t)n2w * nd, L) &&
            alloc_into(h, dc_d, 2 * nd, L) && alloc_into(h, u_d, nd2 * nd2, L) &&
            alloc_into(h, ut_d, nd2 * nd2, L) && alloc_into(h, nd_d, nd, L) &&
            alloc_into(h, gt, (size_t)c.nnu * c.nkp * nd2, L) && alloc_into(h, qd, c.nqp, L) &&
            alloc_into(h, kq, (size_t)c.nkp * c.nqp, L) && alloc_into(h, kqe, (size_t)c.nkp_eom * c.nqp, L);
  if (ok && k_data_eom) ok = alloc_into(h, kde, c.nkp_eom, L);
  if (!ok) { adga_destroy(h); return ADGA_ENOMEM; }
  std::vector<z64> dcz(2 * nd, make_double2(0.0, 0.0));
  if (dc) memcpy(dcz.data(), dc, sizeof(z64) * 2 * nd);
  cudaStream_t st = h->st;
#define UP(dst, src, n) CK(cudaMemcpyAsync(dst, src, (n), cudaMemcpyHostToDevice, st))
  UP(iw, iw_data, sizeof(double) * n2w);
  UP(hk_d, hk, sizeof(z64) * c.nkp * nd2);
  UP(siw_d, siw, sizeof(z64) * n2w * nd);
  UP(giw_d, giw, sizeof(z64) * n2w * nd);
  UP(dc_d, dcz.data(), sizeof(z64) * 2 * nd);
  UP(u_d, u, sizeof(z64) * nd2 * nd2);
  UP(ut_d, u_tilde, sizeof(z64) * nd2 * nd2);
  UP(nd_d, n_dmft, sizeof(z64) * nd);
  UP(qd, q_data, sizeof(int) * c.nqp);
  if (kde) UP(kde, k_data_eom, sizeof(int) * c.nkp_eom);
#undef UP
  c.iw = iw; c.hk = hk_d; c.siw = siw_d; c.giw = giw_d; c.dc = dc_d;
  c.u = u_d; c.ut = ut_d; c.ndmft = nd_d; c.kq = kq; c.kqe = kqe; c.gtab = gt; c.keom = kde;
  CK(launch_kq_index(c.nkpx, c.nkpy, c.nkpz, nullptr, c.nkp, qd, c.nqp, 0, kq, st));
  if (c.nkp_eom == c.nkp && !kde)
    CK(cudaMemcpyAsync(kqe, kq, sizeof(int) * c.nkp * c.nqp, cudaMemcpyDeviceToDevice, st));
  else
    CK(launch_kq_index(c.nkpx, c.nkpy, c.nkpz, kde, c.nkp_eom, qd, c.nqp, 0, kqe, st));
  CK(launch_gtable(c, gt, st));
  if (int rd = setup_dft(h, q_data)) { adga_destroy(h); return rd; }
  // per-omega local buffers and accumulators
  const size_t N = c.N;
  ok = alloc_into(h, h->c0inv, N, L) && alloc_into(h, h->c0w, N, L) &&
       alloc_into(h, h->bubtmp, nd2 * nd2, L) && alloc_into(h, h->Frow_d, N * N, L) &&
       alloc_into(h, h->Frow_m, N * N, L) && alloc_into(h, h->gam_d, nd2 * N, L) &&
       alloc_into(h, h->gam_m, nd2 * N, L) && alloc_into(h, h->opg_d, nd2 * N, L) &&
       alloc_into(h, h->opg_m, nd2 * N, L) && alloc_into(h, h->Frow32_m, N * N, L) &&
       alloc_into(h, h->bubble_loc, (size_t)h->nd4 * h->nw, L) &&
       alloc_into(h, h->chi_loc_d, (size_t)h->nd4 * h->nw, L) &&
       alloc_into(h, h->chi_loc_m, (size_t)h->nd4 * h->nw, L) &&
       alloc_into(h, h->sigma_nl, (size_t)nd2 * 2 * c.iwf * c.nkp_eom, L) &&
       alloc_into(h, h->sigma_dmft, (size_t)nd2 * 2 * c.iwf, L) &&
       alloc_into(h, h->sigma_hf, (size_t)nd2 * c.nkp_eom, L);
  if (!ok) { adga_destroy(h); return ADGA_ENOMEM; }
  h->vd.assign(h->nw, nullptr);
  h->vm.assign(h->nw, nullptr);
  h->tl_d.assign(h->nw, nullptr);
  h->tl_m.assign(h->nw, nullptr);
  CK(cudaStreamSynchronize(st));
  *out = h;
  return adga_reset_outputs(h);
}

extern "C" int adga_destroy(adga_handle *h) {
  if (!h) return 0;
  if (h->st) cudaStreamSynchronize(h->st);
  if (h->tc) tc_trail_free(h->tc);
  if (h->ri8) ri8_free(h->ri8);
  free_list(h->work);
  free_list(h->owned);
  for (auto p : h->vd) if (p) cudaFree(p);
  for (auto p : h->vm) if (p) cudaFree(p);
  if (h->g4buf) cudaFree(h->g4buf);
  for (auto p : h->tl_d) if (p) cudaFree(p);
  for (auto p : h->tl_m) if (p) cudaFree(p);
  if (h->ext_cld) cudaFree(h->ext_cld);
  if (h->ext_clm) cudaFree(h->ext_clm);
  if (h->vq_d) cudaFree(h->vq_d);
  if (h->nfock_d) cudaFree(h->nfock_d);
  if (h->vq_extra) cudaFree(h->vq_extra);
  tan_free(h);
  if (h->qidx_h) cudaFreeHost(h->qidx_h);
  if (h->e0) cudaEventDestroy(h->e0);
  if (h->e1) cudaEventDestroy(h->e1);
  if (h->fork) cudaEventDestroy(h->fork);
  if (h->join) cudaEventDestroy(h->join);
  if (h->st2) { cudaStreamSynchronize(h->st2); cudaStreamDestroy(h->st2); }
  if (h->st) cudaStreamDestroy(h->st);
  delete h;
  return 0;
}

extern "C" int adga_device_bytes(const adga_handle *h, long long *bytes) {
  if (!h || !bytes) return ADGA_EINVAL;
  size_t f = 0, t = 0;
  cudaMemGetInfo(&f, &t);
  *bytes = (long long)(t - f);
  return 0;
}

extern "C" int adga_reset_outputs(adga_handle *h) {
  if (!h) return ADGA_EINVAL;
  const DevCtx &c = h->c;
  cudaStream_t st = h->st;
  CK(cudaMemsetAsync(h->bubble_loc, 0, sizeof(z64) * h->nd4 * h->nw, st));
  CK(cudaMemsetAsync(h->chi_loc_d, 0, sizeof(z64) * h->nd4 * h->nw, st));
  CK(cudaMemsetAsync(h->chi_loc_m, 0, sizeof(z64) * h->nd4 * h->nw, st));
  CK(cudaMemsetAsync(h->sigma_nl, 0, sizeof(z64) * c.nd2 * 2 * c.iwf * c.nkp_eom, st));
  CK(cudaMemsetAsync(h->sigma_dmft, 0, sizeof(z64) * c.nd2 * 2 * c.iwf, st));
  CK(cudaMemsetAsync(h->sigma_hf, 0, sizeof(z64) * c.nd2 * c.nkp_eom, st));
  for (TanState *t : h->tan) {
    if (!t) continue;
    CK(cudaMemsetAsync(t->chi_loc_d, 0, sizeof(z64) * h->nd4 * h->nw, st));
    CK(cudaMemsetAsync(t->chi_loc_m, 0, sizeof(z64) * h->nd4 * h->nw, st));
    CK(cudaMemsetAsync(t->sigma_nl, 0, sizeof(z64) * c.nd2 * 2 * c.iwf * c.nkp_eom, st));
    CK(cudaMemsetAsync(t->sigma_dmft, 0, sizeof(z64) * c.nd2 * 2 * c.iwf, st));
  }
  CK(cudaStreamSynchronize(st));
  return 0;
}

extern "C" int adga_set_vertex(adga_handle *h, int iwb, const adga_z *chi_d, const adga_z *chi_m) {
  if (!h || !chi_d || !chi_m) return ADGA_EINVAL;
  if (iwb < -h->c.iwb || iwb > h->c.iwb) return fail(h, ADGA_EINVAL, "iwb out of range");
  const int w = iwb + h->c.iwb;
  const size_t n = (size_t)h->c.N * h->c.N;
  if (!h->vd[w]) {
    if (cudaMalloc(&h->vd[w], n * sizeof(z64)) != cudaSuccess) return fail(h, ADGA_ENOMEM, "vertex alloc");
    if (cudaMalloc(&h->vm[w], n * sizeof(z64)) != cudaSuccess) return fail(h, ADGA_ENOMEM, "vertex alloc");
  }
  CK(cudaMemcpyAsync(h->vd[w], chi_d, n * sizeof(z64), cudaMemcpyHostToDevice, h->st));
  CK(cudaMemcpyAsync(h->vm[w], chi_m, n * sizeof(z64), cudaMemcpyHostToDevice, h->st));
  if (h->loc_iwb == iwb) h->loc_iwb = INT_MIN;
  CK(cudaStreamSynchronize(h->st));
  return 0;
}

// ---------------------------------------------------------------------------
// index2cor (src/aux.f90:190-221): the correlated bands of atom ineq start
// after all bands of the atoms before it; ndims(nineq, 2) in Fortran order
static int make_atoms(adga_handle *h, int nineq, const int *ndims, VertexAtoms *atoms, const char *who) {
  if (!ndims || nineq < 1) return fail(h, ADGA_EINVAL, std::string(who) + ": missing ndims");
  if (h->c.nd > ADGA_MAX_BANDS) return fail(h, ADGA_EINVAL, std::string(who) + ": more than ADGA_MAX_BANDS bands");
  *atoms = VertexAtoms{};
  int start = 0;
  for (int q = 0; q < nineq; ++q) {
    const int ncor = ndims[q], nunc = ndims[nineq + q];
    if (ncor < 0 || nunc < 0) return fail(h, ADGA_EINVAL, std::string(who) + ": negative band count");
    for (int b = start; b < start + ncor && b < h->c.nd; ++b) atoms->a[b] = q + 1;
    start += ncor + nunc;
  }
  if (start != h->c.nd) return fail(h, ADGA_EINVAL, std::string(who) + ": ndims do not add up to ndim");
  return 0;
}

// upload two host arrays of n elements into the staging buffer (grown on demand)
static int stage_pair(adga_handle *h, const adga_z *a, const adga_z *b, size_t n, const char *who) {
  if (h->g4cap < n) {
    if (h->g4buf) cudaFree(h->g4buf);
    h->g4buf = nullptr;
    h->g4cap = 0;
    if (cudaMalloc(&h->g4buf, 2 * n * sizeof(z64)) != cudaSuccess)
      return fail(h, ADGA_ENOMEM, std::string(who) + ": staging buffer");
    h->g4cap = n;
  }
  CK(cudaMemcpyAsync(h->g4buf, a, n * sizeof(z64), cudaMemcpyHostToDevice, h->st));
  CK(cudaMemcpyAsync(h->g4buf + n, b, n * sizeof(z64), cudaMemcpyHostToDevice, h->st));
  return 0;
}

// vertex ingest (read_vertex's transform, k_vertex.cu)
static int vertex_g4(adga_handle *h, int iwb, int vtype, int W, int nineq, const int *ndims,
                     const adga_z *g4d, const adga_z *g4m, z64 *outd, z64 *outm) {
  const DevCtx &c = h->c;
  if (!g4d || !g4m) return fail(h, ADGA_EINVAL, "vertex_g4: missing argument");
  if (vtype < ADGA_VERTEX_FULL_G4 || vtype > ADGA_VERTEX_CHI_G4)
    return fail(h, ADGA_EINVAL, "vertex_g4: unknown vertex type");
  if (iwb < -c.iwb || iwb > c.iwb) return fail(h, ADGA_EINVAL, "vertex_g4: iwb out of range");
  if (W < c.iwf) return fail(h, ADGA_EINVAL, "vertex_g4: iwfmax_g4 smaller than iwfmax_small");
  VertexAtoms atoms{};
  int r = make_atoms(h, nineq, ndims, &atoms, "vertex_g4");
  if (r) return r;
  const size_t n = (size_t)c.nd2 * c.nd2 * (2 * (size_t)W) * (2 * (size_t)W);
  if ((r = stage_pair(h, g4d, g4m, n, "vertex_g4"))) return r;
  CK(launch_vertex_g4(c, iwb, vtype, W, atoms, h->g4buf, h->g4buf + n, outd, outm, h->st));
  return 0;
}

extern "C" int adga_set_vertex_g4(adga_handle *h, int iwb, int vertex_type, int iwfmax_g4, int nineq,
                                  const int *ndims, const adga_z *g4_dens, const adga_z *g4_magn) {
  if (!h) return ADGA_EINVAL;
  if (iwb < -h->c.iwb || iwb > h->c.iwb) return fail(h, ADGA_EINVAL, "iwb out of range");
  const int w = iwb + h->c.iwb;
  const size_t n = (size_t)h->c.N * h->c.N;
  if (!h->vd[w]) {
    if (cudaMalloc(&h->vd[w], n * sizeof(z64)) != cudaSuccess) return fail(h, ADGA_ENOMEM, "vertex alloc");
    if (cudaMalloc(&h->vm[w], n * sizeof(z64)) != cudaSuccess) return fail(h, ADGA_ENOMEM, "vertex alloc");
  }
  int r = vertex_g4(h, iwb, vertex_type, iwfmax_g4, nineq, ndims, g4_dens, g4_magn, h->vd[w], h->vm[w]);
  if (r) return r;
  if (h->loc_iwb == iwb) h->loc_iwb = INT_MIN;
  CK(cudaStreamSynchronize(h->st));
  return 0;
}

extern "C" int adga_vertex_transform(adga_handle *h, int iwb, int vertex_type, int iwfmax_g4, int nineq,
                                     const int *ndims, const adga_z *g4_dens, const adga_z *g4_magn,
                                     adga_z *chi_loc_dens, adga_z *chi_loc_magn) {
  if (!h || !chi_loc_dens || !chi_loc_magn) return ADGA_EINVAL;
  const size_t n = (size_t)h->c.N * h->c.N;
  z64 *tmp = nullptr;
  if (cudaMalloc(&tmp, 2 * n * sizeof(z64)) != cudaSuccess) return fail(h, ADGA_ENOMEM, "transform output");
  int r = vertex_g4(h, iwb, vertex_type, iwfmax_g4, nineq, ndims, g4_dens, g4_magn, tmp, tmp + n);
  if (!r && (cudaMemcpyAsync(chi_loc_dens, tmp, n * sizeof(z64), cudaMemcpyDeviceToHost, h->st) != cudaSuccess ||
             cudaMemcpyAsync(chi_loc_magn, tmp + n, n * sizeof(z64), cudaMemcpyDeviceToHost, h->st) != cudaSuccess ||
             cudaStreamSynchronize(h->st) != cudaSuccess))
    r = fail(h, ADGA_ECUDA, "transform download");
  cudaFree(tmp);
  return r;
}

extern "C" int adga_index2component_band(int nbands, int ind, int *b) {
  if (!b || nbands < 1 || ind < 1 || ind > nbands * nbands * nbands * nbands) return ADGA_EINVAL;
  const int i = ind - 1, n3 = nbands * nbands * nbands, n2 = nbands * nbands;
  b[0] = i / n3 + 1;
  b[1] = (i % n3) / n2 + 1;
  b[2] = (i % n2) / nbands + 1;
  b[3] = i % nbands + 1;
  return 0;
}

extern "C" int adga_set_threeleg(adga_handle *h, int iwb, int n3iwf, int nineq, const int *ndims,
                                 const adga_z *g3_dens, const adga_z *g3_magn) {
  if (!h || !g3_dens || !g3_magn) return ADGA_EINVAL;
  const DevCtx &c = h->c;
  if (iwb < -c.iwb || iwb > c.iwb) return fail(h, ADGA_EINVAL, "set_threeleg: iwb out of range");
  if (n3iwf < c.iwf) return fail(h, ADGA_EINVAL, "set_threeleg: n3iwf smaller than iwfmax_small");
  VertexAtoms atoms{};
  int r = make_atoms(h, nineq, ndims, &atoms, "set_threeleg");
  if (r) return r;
  const int w = iwb + c.iwb;
  const size_t ng = (size_t)c.nd2 * c.N;
  if (!h->tl_d[w]) {
    if (cudaMalloc(&h->tl_d[w], ng * sizeof(z64)) != cudaSuccess ||
        cudaMalloc(&h->tl_m[w], ng * sizeof(z64)) != cudaSuccess)
      return fail(h, ADGA_ENOMEM, "set_threeleg: gamma storage");
  }
  const size_t n = (size_t)c.nd2 * c.nd2 * 2 * (size_t)n3iwf;
  if ((r = stage_pair(h, g3_dens, g3_magn, n, "set_threeleg"))) return r;
  CK(launch_threeleg(c, iwb, n3iwf, atoms, h->g4buf, h->g4buf + n, h->tl_d[w], h->tl_m[w], h->st));
  if (h->loc_iwb == iwb) h->loc_iwb = INT_MIN;
  CK(cudaStreamSynchronize(h->st));
  return 0;
}

extern "C" int adga_set_chi_loc_ext(adga_handle *h, int n2iwb, int nineq, const int *ndims,
                                    const adga_z *chi_dens, const adga_z *chi_magn) {
  if (!h || !chi_dens || !chi_magn) return ADGA_EINVAL;
  const DevCtx &c = h->c;
  if (n2iwb < c.iwb) return fail(h, ADGA_EINVAL, "set_chi_loc_ext: n2iwb smaller than iwbmax_small");
  VertexAtoms atoms{};
  int r = make_atoms(h, nineq, ndims, &atoms, "set_chi_loc_ext");
  if (r) return r;
  const size_t nc = (size_t)h->nd4 * h->nw;
  if (!h->ext_cld) {
    if (cudaMalloc(&h->ext_cld, nc * sizeof(z64)) != cudaSuccess ||
        cudaMalloc(&h->ext_clm, nc * sizeof(z64)) != cudaSuccess)
      return fail(h, ADGA_ENOMEM, "set_chi_loc_ext: storage");
  }
  const size_t n = (size_t)h->nd4 * (2 * (size_t)n2iwb + 1);
  if ((r = stage_pair(h, chi_dens, chi_magn, n, "set_chi_loc_ext"))) return r;
  // read_chi_loc extends the bubble unless one impurity holds every band as correlated
  const int extend = !(ndims[0] == c.nd);
  CK(launch_chi_loc_ext(c, n2iwb, atoms, extend, h->g4buf, h->g4buf + n, h->ext_cld, h->ext_clm, h->st));
  CK(cudaStreamSynchronize(h->st));
  return 0;
}

extern "C" int adga_set_vq(adga_handle *h, const adga_z *vq) {
  if (!h) return ADGA_EINVAL;
  DevCtx &c = h->c;
  if (!vq) {                    // switch the non-local interaction off
    c.vq = nullptr;
    c.nfock = nullptr;
    h->loc_iwb = INT_MIN;
    return 0;
  }
  if (c.nd > GINV_MAXND_HOST) return fail(h, ADGA_EINVAL, "set_vq: ndim above 8");
  const size_t nv = (size_t)h->nd4 * c.nqp;
  if (!h->vq_d) {
    if (cudaMalloc(&h->vq_d, nv * sizeof(z64)) != cudaSuccess ||
        cudaMalloc(&h->nfock_d, (size_t)c.nkp * c.nd2 * sizeof(z64)) != cudaSuccess)
      return fail(h, ADGA_ENOMEM, "set_vq: storage");
  }
  z64 *raw = nullptr;
  if (cudaMalloc(&raw, nv * sizeof(z64)) != cudaSuccess) return fail(h, ADGA_ENOMEM, "set_vq: staging");
  cudaError_t e = cudaMemcpyAsync(raw, vq, nv * sizeof(z64), cudaMemcpyHostToDevice, h->st);
  if (e == cudaSuccess) e = launch_vq_permute(c.nd, c.nqp, raw, h->vq_d, h->st);
  if (e == cudaSuccess) e = launch_nfock(c, h->nfock_d, h->st);      // get_nfock
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->st);
  cudaFree(raw);
  if (e != cudaSuccess) return fail(h, ADGA_ECUDA, std::string("set_vq: ") + cudaGetErrorString(e));
  c.vq = h->vq_d;
  c.nfock = h->nfock_d;
  h->loc_iwb = INT_MIN;
  return 0;
}

// ---------------------------------------------------------------------------
static int ensure_diag(adga_handle *h, int iwb) {
  if (h->diag_iwb == iwb) return 0;
  CK(launch_local_diag(h->c, iwb, h->c0inv, h->c0w, h->bubtmp, h->st));
  h->diag_iwb = iwb;
  h->loc_iwb = INT_MIN;
  return 0;
}

// src/main.F90:506-627 for omega = iwb
static int ensure_local(adga_handle *h, int iwb) {
  if (h->loc_iwb == iwb) return 0;
  const int w = iwb + h->c.iwb;
  if (!h->vd[w]) return fail(h, ADGA_ESTATE, "vertex of omega " + std::to_string(iwb) + " not set");
  int r = ensure_diag(h, iwb);
  if (r) return r;
  CK(launch_local_F(h->c, h->vd[w], h->c0inv, h->Frow_d, h->st));
  CK(launch_local_F(h->c, h->vm[w], h->c0inv, h->Frow_m, h->st));
  h->f32_iwb = INT_MIN;
  ++h->frow_gen;
  if (h->tl_d[w]) {
    // external three-leg vertex (src/main.F90:560-561), then 1 + gamma^w
    const size_t ng = (size_t)h->c.nd2 * h->c.N;
    CK(cudaMemcpyAsync(h->gam_d, h->tl_d[w], ng * sizeof(z64), cudaMemcpyDeviceToDevice, h->st));
    CK(cudaMemcpyAsync(h->gam_m, h->tl_m[w], ng * sizeof(z64), cudaMemcpyDeviceToDevice, h->st));
    CK(launch_one_plus_gamma(h->c, h->gam_d, h->opg_d, h->st));
    CK(launch_one_plus_gamma(h->c, h->gam_m, h->opg_m, h->st));
  } else {
    CK(launch_local_gamma(h->c, h->Frow_d, h->gam_d, h->opg_d, h->st));
    CK(launch_local_gamma(h->c, h->Frow_m, h->gam_m, h->opg_m, h->st));
  }
  h->loc_iwb = iwb;
  return 0;
}

static size_t bytes_per_point(const adga_handle *h, int prec, int NB) {
  const DevCtx &c = h->c;
  const size_t N = c.N, R = c.R, nd2 = c.nd2;
  const size_t nsteps = (N + NB - 1) / NB;
  size_t b = 0;
  b += h->nd4 * (size_t)h->nnu_all * 16 + (h->bigbox ? h->nd4 * 2 * c.iwf * 16 : 0);
  b += 3 * nd2 * N * 16 + nd2 * c.iwf * nd2 * 16 + 2 * N * 4 + 16;
  if (prec == ADGA_FP64) {
    b += 2 * N * (N + R) * 16 + 2 * 2 * nsteps * NB * NB * 16;
  } else {
    b += 2 * N * (N + R) * 8 + 2 * 2 * nsteps * NB * NB * 8;
    b += 2 * 2 * R * N * 16 + 2 * R * N * 8 + 2 * ((R + 15) / 16) * 16 * N * 8 + 2 * N * 4 + 64;
    b += 2 * 7 * R * ((2 * N + 63) / 64 * 64) + 2 * R * 4;   // int8 residual slices and scales
    b += 2 * 4 * (N + N + R) * 4 * NB * 2;                     // four tensor-core operand stagings
  }
  return b;
}

static int ensure_work(adga_handle *h, int prec, int want) {
  const DevCtx &c = h->c;
  if (h->tune.batch > 0) want = std::min(want, h->tune.batch);
  if (h->cap_prec == prec && h->cap >= want && (h->tune.batch <= 0 || h->cap <= h->tune.batch)) return 0;
  cudaStreamSynchronize(h->st);
  if (h->tc) { tc_trail_free(h->tc); h->tc = nullptr; }
  if (h->ri8) { ri8_free(h->ri8); h->ri8 = nullptr; }
  free_list(h->work);
  h->cap = 0;
  h->cap_prec = -1;
  const int NB = prec == ADGA_FP64 ? 64 : h->NB;
  size_t per = bytes_per_point(h, prec, NB);
  size_t fr = 0, tot = 0;
  cudaMemGetInfo(&fr, &tot);
  double frac = h->tan_on ? 0.3 : 0.6;   // tangent runs hold about as much again
  const char *e = getenv("ADGA_WORK_FRAC");
  if (e) frac = atof(e);
  size_t budget = (size_t)(fr * frac);
  int cap = (int)std::min<size_t>((size_t)want, std::max<size_t>(1, budget / per));
  const char *eb = getenv("ADGA_BATCH");
  if (eb) cap = std::max(1, std::min(cap, atoi(eb)));
  const size_t N = c.N, R = c.R, nd2 = c.nd2, nsteps = (N + NB - 1) / NB;
  auto &W = h->work;
  bool ok = alloc_into(h, h->chi0_all, (size_t)cap * h->nd4 * h->nnu_all, W) &&
            alloc_into(h, h->gq, (size_t)cap * nd2 * N, W) &&
            alloc_into(h, h->mtot, (size_t)cap * nd2 * c.iwf * nd2, W) &&
            alloc_into(h, h->etad, (size_t)cap * nd2 * N, W) &&
            alloc_into(h, h->etam, (size_t)cap * nd2 * N, W) &&
            alloc_into(h, h->qidx_d, cap, W) && alloc_into(h, h->ipiv, (size_t)2 * cap * N, W) &&
            alloc_into(h, h->info, (size_t)2 * cap, W) &&
            alloc_into(h, h->rmap, (size_t)2 * cap * RMAP_STRIDE, W);
  if (ok && h->bigbox) ok = alloc_into(h, h->chi0q_big, (size_t)cap * h->nd4 * 2 * c.iwf, W);
  if (ok) {
    const size_t es = prec == ADGA_FP64 ? 16 : 8;
    h->Tm = dalloc(h, (size_t)2 * cap * N * (N + R) * es, W);
    h->Linv = dalloc(h, (size_t)2 * cap * nsteps * NB * NB * es, W);
    h->Uinv = dalloc(h, (size_t)2 * cap * nsteps * NB * NB * es, W);
    ok = h->Tm && h->Linv && h->Uinv;
  }
  if (ok && prec == ADGA_MIXED) {
    ok = alloc_into(h, h->X64, (size_t)2 * cap * R * N, W) &&
         alloc_into(h, h->XD, (size_t)2 * cap * R * N, W) &&
         alloc_into(h, h->V32, (size_t)2 * cap * R * N, W) &&
         alloc_into(h, h->work32, (size_t)2 * cap * ((R + 15) / 16) * 16 * N, W) &&
         alloc_into(h, h->perm, (size_t)2 * cap * N, W) &&
         alloc_into(h, h->norms, (size_t)6 * cap, W);   // [max|d|, max|X|] per matrix, then max|r|
  }
  if (!ok) {
    free_list(h->work);
    return fail(h, ADGA_ENOMEM, "batch work buffers (" + std::to_string(cap) + " points)");
  }
  if (h->qidx_h) cudaFreeHost(h->qidx_h);
  CK(cudaMallocHost(&h->qidx_h, sizeof(int) * cap));
  h->cap = cap;
  h->cap_prec = prec;
  if (prec == ADGA_MIXED && tc_available() && !getenv("ADGA_NO_TC")) {
    LUBatch lb{(int)N, (int)(N + R), 2 * cap, NB, N * (N + R), h->ipiv, h->info, h->Linv, h->Uinv, h->rmap};
    if (tc_trail_setup(&h->tc, (z32 *)h->Tm, lb, h->st) != cudaSuccess) h->tc = nullptr;
    // the int8-slice residual (its slices and maps for this batch size)
    if (ri8_setup(&h->ri8, (int)N, (int)R, cap) != cudaSuccess) h->ri8 = nullptr;
  }
  return 0;
}

static void stage_ms(adga_handle *h, double *acc, cudaEvent_t a, cudaEvent_t b) {
  float ms = 0.f;
  if (cudaEventElapsedTime(&ms, a, b) == cudaSuccess) *acc += ms;
}

// LU of the whole batch.  Optionally (ADGA_TWO_STREAMS) the batch is split in
// halves whose steps are issued alternately on two streams, so that the
// latency-bound phases of one half (panel, block inverses, interchanges) can
// overlap the trailing updates of the other.  Timing events bracket the
// (first half's) trailing updates.
template <typename T>
static cudaError_t factor_batch(adga_handle *h, T *M, const LUBatch &lb, bool apply_left, bool tc,
                                TrailTiming *tt, bool nopiv = false) {
  cudaStream_t st = h->st;
  // measured: the trailing-update grids fill every SM, so the split gives no
  // overlap on the t2g workload; kept as an option (ADGA_TWO_STREAMS=1)
  const bool split = h->st2 && lb.batch >= 8 && getenv("ADGA_TWO_STREAMS");
  if constexpr (sizeof(T) == sizeof(z32)) {
    // unpivoted FP32 with the tensor cores: delayed updates in groups of tune.pairs + 1 steps
    // (tune.pairs = 0: step by step)
    if (!split && nopiv && tc && tc_pair_supported(h->tc) && h->tune.pairs) {
      // L21 / U12 on the tensor cores with the staging written by the same kernel
      // (tune.tri_tc = 0: the FP32 CUDA-core tile products and the split kernels)
      const bool tri_tc = (lb.N % 2) == 0 && h->tune.tri_tc;
      TcRange r{h->tc, 0, lb.batch, tri_tc};
      GroupOps ops{tc_group_fn, &r, tri_tc ? tc_tri_fn : nullptr, h->tune.pairs + 1};
      return lu_factor_groups(M, lb, ops, st, tt);
    }
  }
  if (!split) {
    TcRange r{h->tc, 0, lb.batch};
    return lu_factor<T>(M, lb, apply_left, tc ? tc_trail_range_fn : nullptr, tc ? &r : nullptr, st, tt, nopiv);
  }
  const int na = lb.batch / 2, nb = lb.batch - na;
  LUBatch la = lu_sub<T>(lb, 0, na), lbb = lu_sub<T>(lb, na, nb);
  T *Mb = M + (size_t)na * lb.strideM;
  TcRange ra{h->tc, 0, na}, rb{h->tc, na, nb};
  cudaError_t e = cudaEventRecord(h->fork, st);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(h->st2, h->fork, 0);
  for (int s = 0; e == cudaSuccess && s < lb.nsteps(); ++s) {
    e = lu_step<T>(M, la, s, apply_left, tc ? tc_trail_range_fn : nullptr, tc ? &ra : nullptr, st, tt, nopiv);
    if (e == cudaSuccess)
      e = lu_step<T>(Mb, lbb, s, apply_left, tc ? tc_trail_range_fn : nullptr, tc ? &rb : nullptr, h->st2,
                     nullptr, nopiv);
  }
  if (e == cudaSuccess) e = cudaEventRecord(h->join, h->st2);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(st, h->join, 0);
  return e;
}

// one batch of np consecutive q at omega = iwb: chi0 -> build -> LU/solve -> post -> EOM.
// qidx_h[0..np) hold the 0-based q indices; outputs go to point slot `off`.
// ---------------------------------------------------------------------------
// Tangent (forward-mode) ladder: derivatives of the FP64 outputs along one
// parameter direction, given the direction's dH(k), du, du~ and dchi_loc(omega)
// (k_tangent.cu has the BSE algebra; every other stage reuses the forward
// kernels with swapped pointers, since they are linear in each argument).
// ---------------------------------------------------------------------------

static bool tan_dir_ok(int d) { return d >= 0 && d < ADGA_MAX_TANGENTS; }

// shared constants of the tangent passes
static int tan_shared(adga_handle *h) {
  if (h->tw) return 0;
  const DevCtx &c = h->c;
  TanWork *w = new TanWork();
  h->tw = w;
  const size_t N = c.N, nd2 = c.nd2;
  auto &L = w->owned;
  if (!(alloc_into(h, w->zero_nd4, nd2 * nd2, L) && alloc_into(h, w->zero_N, N, L) &&
        alloc_into(h, w->zero_gam, nd2 * N, L) && alloc_into(h, w->opg_scr, nd2 * N, L) &&
        alloc_into(h, w->bub_scr, nd2 * nd2, L)))
    return fail(h, ADGA_ENOMEM, "tangent constants");
  CK(cudaMemsetAsync(w->zero_nd4, 0, sizeof(z64) * nd2 * nd2, h->st));
  CK(cudaMemsetAsync(w->zero_N, 0, sizeof(z64) * N, h->st));
  CK(cudaMemsetAsync(w->zero_gam, 0, sizeof(z64) * nd2 * N, h->st));
  return 0;
}

static int tan_state(adga_handle *h, int d) {
  int r = tan_shared(h);
  if (r) return r;
  if (h->tan[d]) return 0;
  const DevCtx &c = h->c;
  TanState *t = new TanState();
  h->tan[d] = t;
  t->vd.assign(h->nw, nullptr);
  t->vm.assign(h->nw, nullptr);
  const size_t N = c.N, nd2 = c.nd2, nw = h->nw;
  auto &L = t->owned;
  bool ok = alloc_into(h, t->gdot, (size_t)c.nnu * c.nkp * nd2, L) && alloc_into(h, t->du, nd2 * nd2, L) &&
            alloc_into(h, t->dut, nd2 * nd2, L) && alloc_into(h, t->Fd, N * N, L) &&
            alloc_into(h, t->Fm, N * N, L) && alloc_into(h, t->gd, nd2 * N, L) && alloc_into(h, t->gm, nd2 * N, L) &&
            alloc_into(h, t->chi_loc_d, nd2 * nd2 * nw, L) && alloc_into(h, t->chi_loc_m, nd2 * nd2 * nw, L) &&
            alloc_into(h, t->sigma_nl, nd2 * 2 * c.iwf * (size_t)c.nkp_eom, L) &&
            alloc_into(h, t->sigma_dmft, nd2 * 2 * c.iwf, L);
  if (ok && c.dft.ghat) ok = alloc_into(h, t->ghat_dot, (size_t)c.nnu * c.nkp * nd2, L);
  if (!ok) return fail(h, ADGA_ENOMEM, "tangent direction");
  CK(cudaMemsetAsync(t->du, 0, sizeof(z64) * nd2 * nd2, h->st));
  CK(cudaMemsetAsync(t->dut, 0, sizeof(z64) * nd2 * nd2, h->st));
  CK(cudaMemsetAsync(t->chi_loc_d, 0, sizeof(z64) * nd2 * nd2 * nw, h->st));
  CK(cudaMemsetAsync(t->chi_loc_m, 0, sizeof(z64) * nd2 * nd2 * nw, h->st));
  CK(cudaMemsetAsync(t->sigma_nl, 0, sizeof(z64) * nd2 * 2 * c.iwf * c.nkp_eom, h->st));
  CK(cudaMemsetAsync(t->sigma_dmft, 0, sizeof(z64) * nd2 * 2 * c.iwf, h->st));
  return 0;
}

static void tan_free(adga_handle *h) {
  for (TanState *&t : h->tan) {
    if (!t) continue;
    free_list(t->owned);
    for (auto p : t->vd) if (p) cudaFree(p);
    for (auto p : t->vm) if (p) cudaFree(p);
    for (z64 *p : {t->chi_qw_d, t->chi_qw_m, t->bub_nl}) if (p) cudaFree(p);
    delete t;
    t = nullptr;
  }
  if (h->tw) {
    free_list(h->tw->work);
    free_list(h->tw->owned);
    delete h->tw;
    h->tw = nullptr;
  }
}

extern "C" int adga_set_tangent(adga_handle *h, int dir, const adga_z *dhk, const adga_z *du,
                                const adga_z *du_tilde) {
  if (!h) return ADGA_EINVAL;
  if (!tan_dir_ok(dir)) return fail(h, ADGA_EINVAL, "set_tangent: direction outside 0..ADGA_MAX_TANGENTS-1");
  int r = tan_state(h, dir);
  if (r) return r;
  TanState *t = h->tan[dir];
  const DevCtx &c = h->c;
  const size_t nd4 = (size_t)c.nd2 * c.nd2;
  if (du) CK(cudaMemcpyAsync(t->du, du, sizeof(z64) * nd4, cudaMemcpyHostToDevice, h->st));
  else CK(cudaMemsetAsync(t->du, 0, sizeof(z64) * nd4, h->st));
  if (du_tilde) CK(cudaMemcpyAsync(t->dut, du_tilde, sizeof(z64) * nd4, cudaMemcpyHostToDevice, h->st));
  else CK(cudaMemsetAsync(t->dut, 0, sizeof(z64) * nd4, h->st));
  t->has_dhk = dhk != nullptr;
  if (dhk) {
    z64 *dh = nullptr;
    if (cudaMalloc(&dh, sizeof(z64) * c.nd2 * c.nkp) != cudaSuccess) return fail(h, ADGA_ENOMEM, "dhk");
    cudaError_t e = cudaMemcpyAsync(dh, dhk, sizeof(z64) * c.nd2 * c.nkp, cudaMemcpyHostToDevice, h->st);
    if (e == cudaSuccess) e = launch_gtable_dot(c, dh, t->gdot, h->st);   // dG = G dH G
    if (e == cudaSuccess && t->ghat_dot) e = launch_gtable_dft(c, t->gdot, t->ghat_dot, c.dft.a, h->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->st);
    cudaFree(dh);
    if (e != cudaSuccess) return fail(h, ADGA_ECUDA, "set_tangent: dG table");
  }
  CK(cudaStreamSynchronize(h->st));
  return 0;
}

extern "C" int adga_clear_tangents(adga_handle *h) {
  if (!h) return ADGA_EINVAL;
  cudaStreamSynchronize(h->st);
  tan_free(h);
  return 0;
}

extern "C" int adga_set_vertex_tangent(adga_handle *h, int dir, int iwb, const adga_z *dchi_d,
                                       const adga_z *dchi_m) {
  if (!h) return ADGA_EINVAL;
  if (!tan_dir_ok(dir)) return fail(h, ADGA_EINVAL, "set_vertex_tangent: direction out of range");
  if (iwb < -h->c.iwb || iwb > h->c.iwb) return fail(h, ADGA_EINVAL, "iwb out of range");
  int r = tan_state(h, dir);
  if (r) return r;
  TanState *t = h->tan[dir];
  const int w = iwb + h->c.iwb;
  const size_t n = (size_t)h->c.N * h->c.N;
  t->loc_iwb = INT_MIN;
  if (!dchi_d || !dchi_m) {
    if (t->vd[w]) { cudaFree(t->vd[w]); cudaFree(t->vm[w]); t->vd[w] = t->vm[w] = nullptr; }
    return 0;
  }
  if (!t->vd[w] && (cudaMalloc(&t->vd[w], n * sizeof(z64)) != cudaSuccess ||
                    cudaMalloc(&t->vm[w], n * sizeof(z64)) != cudaSuccess))
    return fail(h, ADGA_ENOMEM, "vertex tangent");
  CK(cudaMemcpyAsync(t->vd[w], dchi_d, n * sizeof(z64), cudaMemcpyHostToDevice, h->st));
  CK(cudaMemcpyAsync(t->vm[w], dchi_m, n * sizeof(z64), cudaMemcpyHostToDevice, h->st));
  CK(cudaStreamSynchronize(h->st));
  return 0;
}

// dF~ and dgamma^w of direction d at omega = iwb (after ensure_local)
static int tan_local(adga_handle *h, int d, int iwb) {
  TanState *t = h->tan[d];
  if (t->loc_iwb == iwb) return 0;
  const int w = iwb + h->c.iwb;
  t->loc_has = t->vd[w] != nullptr;
  if (t->loc_has) {
    // F~ = sym(chi_loc) chi0_loc^-1 - 1 is affine in chi_loc: dF~ = sym(dchi_loc) chi0_loc^-1
    CK(launch_local_F(h->c, t->vd[w], h->c0inv, t->Fd, h->st, false));
    CK(launch_local_F(h->c, t->vm[w], h->c0inv, t->Fm, h->st, false));
    CK(launch_local_gamma(h->c, t->Fd, t->gd, h->tw->opg_scr, h->st));
    CK(launch_local_gamma(h->c, t->Fm, t->gm, h->tw->opg_scr, h->st));
  }
  t->loc_iwb = iwb;
  return 0;
}

static int tan_work(adga_handle *h) {
  TanWork *t = h->tw;
  if (t->cap >= h->cap) return 0;
  free_list(t->work);
  t->cap = 0;
  const DevCtx &c = h->c;
  const size_t cap = h->cap, N = c.N, R = c.R, nd2 = c.nd2, nd4 = (size_t)h->nd4;
  const size_t per = R * N;
  auto &W = t->work;
  bool ok = alloc_into(h, t->chi0_all, cap * nd4 * h->nnu_all, W) &&
            alloc_into(h, t->chi0_tmp, cap * nd4 * h->nnu_all, W) &&
            alloc_into(h, t->zero_chi0, cap * nd4 * 2 * c.iwf, W) && alloc_into(h, t->Xc, 2 * cap * per, W) &&
            alloc_into(h, t->XS, 2 * cap * per, W) && alloc_into(h, t->XD, 2 * cap * per, W) &&
            alloc_into(h, t->Rt, 2 * cap * per, W) && alloc_into(h, t->wk, 2 * cap * ((R + 15) / 16) * 16 * N, W) &&
            alloc_into(h, t->gq, cap * nd2 * N, W) && alloc_into(h, t->cA_d, cap * nd4, W) &&
            alloc_into(h, t->cA_m, cap * nd4, W) && alloc_into(h, t->cB_d, cap * nd4, W) &&
            alloc_into(h, t->cB_m, cap * nd4, W) && alloc_into(h, t->mA, cap * nd2 * c.iwf * nd2, W) &&
            alloc_into(h, t->mB, cap * nd2 * c.iwf * nd2, W) && alloc_into(h, t->eta_d, cap * nd2 * N, W) &&
            alloc_into(h, t->eta_m, cap * nd2 * N, W) && alloc_into(h, t->perm, 2 * cap * N, W);
  if (ok && h->bigbox) ok = alloc_into(h, t->chi0q_big, cap * nd4 * 2 * c.iwf, W);
  if (!ok) return fail(h, ADGA_ENOMEM, "tangent batch buffers");
  CK(cudaMemsetAsync(t->zero_chi0, 0, sizeof(z64) * cap * nd4 * 2 * c.iwf, h->st));
  t->cap = (int)cap;
  return 0;
}

// dX = r A^-1 for the tangents of a mixed batch: the forward pass's FP32
// factors and FP64 refinement against 1 - D F~ with r in place of (1+gamma^w)
// (the residual r - dX + (dX D) F~), the same stopping rules as the forward
// refinement, with up to kTanIterFactor times the forward's sweeps (a tangent's
// relative error starts where the forward's starts, but its right-hand side
// may be small beside the solve's scale, which takes the relative test longer).
// Matrices flagged in skip (points the forward re-solves in FP64) are left out
// of the convergence test.
constexpr int kTanIterFactor = 3;
static int tan_solve_mixed(adga_handle *h, z32 *T, const LUBatch &lb, const z64 *chi0q, int np, const z64 *r,
                           z64 *dX, const std::vector<char> &skip) {
  DevCtx &c = h->c;
  cudaStream_t st = h->st;
  const size_t N = c.N, R = c.R, per = N * R;
  const int nmat = 2 * np;
  unsigned long long *rnorm = h->norms + 4 * (size_t)h->cap;
  std::vector<unsigned long long> nh(3 * nmat);
  std::vector<double> rho(nmat, 1.0), xmax(nmat, 0.0);
  auto bits = [](unsigned long long u) { double x; memcpy(&x, &u, 8); return x; };
  CK(cudaMemsetAsync(dX, 0, sizeof(z64) * nmat * per, st));
  CK(launch_to32((size_t)nmat * per, r, h->V32, st));
  CK(lu_fwdsolve_ws<z32>(T, lb, h->V32, per, (int)N, (int)R, h->work32, st));
  CK(lu_backsolve<z32>(T, lb, h->V32, per, (int)N, (int)R, st));
  CK(cudaMemsetAsync(h->norms, 0, sizeof(unsigned long long) * 2 * nmat, st));
  CK(launch_update((int)per, nmat, h->V32, dX, h->norms, nullptr, st));
  int nbad = 0, wbad = -1;
  double wrel = 0.0;
  for (int it = 0; it < kTanIterFactor * h->max_iter; ++it) {
    CK(cudaMemsetAsync(h->norms, 0, sizeof(unsigned long long) * 2 * nmat, st));
    CK(cudaMemsetAsync(rnorm, 0, sizeof(unsigned long long) * nmat, st));
    CK(launch_residual(c, np, dX, chi0q, h->c0inv, h->Frow_d, h->Frow_m, h->opg_d, h->opg_m, h->XD, h->V32,
                       nullptr, rnorm, st, r, h->tune.resid ? h->ri8 : nullptr, h->frow_gen));
    if (it > 0 && h->refine_estimate) {
      CK(cudaMemcpyAsync(nh.data() + 2 * nmat, rnorm, sizeof(unsigned long long) * nmat, cudaMemcpyDeviceToHost,
                         st));
      CK(cudaStreamSynchronize(st));
      bool all = true;
      for (int m = 0; m < nmat && all; ++m) {
        if (skip[m]) continue;
        const double est = kEstSafety * std::max(rho[m], 1.0) * bits(nh[2 * nmat + m]);
        if (!((xmax[m] > 0 ? est / xmax[m] : est) <= h->tol)) all = false;
      }
      if (all) {
        h->stats.max_refine_iters = std::max(h->stats.max_refine_iters, it + 1);
        return 0;
      }
    }
    CK(lu_fwdsolve_ws<z32>(T, lb, h->V32, per, (int)N, (int)R, h->work32, st));
    CK(lu_backsolve<z32>(T, lb, h->V32, per, (int)N, (int)R, st));
    CK(launch_update((int)per, nmat, h->V32, dX, h->norms, nullptr, st));
    CK(cudaMemcpyAsync(nh.data(), h->norms, sizeof(unsigned long long) * 2 * nmat, cudaMemcpyDeviceToHost, st));
    if (it == 0)
      CK(cudaMemcpyAsync(nh.data() + 2 * nmat, rnorm, sizeof(unsigned long long) * nmat, cudaMemcpyDeviceToHost,
                         st));
    CK(cudaStreamSynchronize(st));
    nbad = 0;
    wbad = -1;
    wrel = 0.0;
    for (int m = 0; m < nmat; ++m) {
      const double md = bits(nh[2 * m]), mx = bits(nh[2 * m + 1]);
      xmax[m] = mx;
      if (it == 0) {
        const double r1 = bits(nh[2 * nmat + m]);
        rho[m] = r1 > 0 ? md / r1 : 1.0;
      }
      const double rel = mx > 0 ? md / mx : md;
      if (!skip[m] && !(rel <= h->tol)) {
        ++nbad;
        if (!(rel <= wrel)) { wrel = rel; wbad = m; }
      }
    }
    if (!nbad) {
      // the run's refinement statistics cover the tangent solves too
      h->stats.max_refine_iters = std::max(h->stats.max_refine_iters, it + 1);
      return 0;
    }
  }
  char msg[256];
  snprintf(msg, sizeof msg,
           "tangent refinement did not converge: %d of %d matrices after %d sweeps (worst: matrix %d, "
           "max|correction| / max|dX| = %.3g, max|dX| = %.3g, first-sweep amplification %.3g)",
           nbad, nmat, kTanIterFactor * h->max_iter, wbad, wrel, wbad >= 0 ? xmax[wbad] : 0.0,
           wbad >= 0 ? rho[wbad] : 0.0);
  return fail(h, ADGA_ENOCONV, msg);
}

// the tangent of direction d for one batch, after its forward pass.  FP64: T holds
// the LU factors of the transposed BSE matrices (factorised with the left
// interchanges) and X sits beside them; mixed: T holds the FP32 factors, X is
// the refined X64, and the points in skip are re-solved in FP64 (with their
// tangents) after this batch, so their tangent EOM terms are left out here.
static int tan_batch(adga_handle *h, int d, int iwb, int np, int off, void *Tv, LUBatch lb, const z64 *chi0q,
                     bool do_chi, bool do_eom, bool mixed, const std::vector<int> &skip) {
  TanState *t = h->tan[d];
  DevCtx &c = h->c;
  cudaStream_t st = h->st;
  const size_t N = c.N, R = c.R, per = R * N, strideM = N * (N + R);
  int r = tan_work(h);
  if (r) return r;
  TanWork *w = h->tw;
  // dchi0^q = -(beta/nkp) sum_k [dG(k) G(k-q) + G(k) dG(k-q)]
  const z64 *dchi0q = nullptr;
  if (t->has_dhk) {
    DevCtx cg = c;
    cg.gtab = t->gdot;
    cg.dft.ghat = t->ghat_dot;
    CK(launch_chi0(cg, iwb, h->qidx_d, np, w->chi0_all, h->nnu_all, st, c.gtab, c.dft.ghat));
    CK(launch_chi0(c, iwb, h->qidx_d, np, w->chi0_tmp, h->nnu_all, st, t->gdot, t->ghat_dot));
    CK(launch_zadd((size_t)np * h->nd4 * h->nnu_all, w->chi0_tmp, w->chi0_all, st));
    dchi0q = h->bigbox ? w->chi0q_big : w->chi0_all;
    CK(launch_chi0_finish(c, w->chi0_all, h->nnu_all, np, w->zero_nd4, h->bigbox ? w->chi0q_big : nullptr,
                          do_chi ? t->bub_nl + (size_t)off * h->nd4 : nullptr, st));
  }
  // X (compact) and the tangent right-hand sides dB + XS F~ + XD dF~
  z64 *T = (z64 *)Tv;
  const z64 *Xp = mixed ? h->X64 : w->Xc;
  if (!mixed)
    CK(cudaMemcpy2DAsync(w->Xc, per * sizeof(z64), T + N * N, strideM * sizeof(z64), per * sizeof(z64), 2 * np,
                         cudaMemcpyDeviceToDevice, st));
  CK(launch_xd(c, np, Xp, chi0q, h->c0inv, w->XD, true, st));
  if (dchi0q) CK(launch_xd(c, np, Xp, dchi0q, h->c0inv, w->XS, false, st));
  for (int ch = 0; ch < 2; ++ch)
    CK(launch_tan_rhs(c, np, ch, dchi0q ? w->XS : nullptr, ch ? h->Frow_m : h->Frow_d,
                      t->loc_has ? w->XD : nullptr, t->loc_has ? (ch ? t->Fm : t->Fd) : nullptr,
                      t->loc_has ? (ch ? t->gm : t->gd) : nullptr, w->Rt, st));
  // dX = r A^-1 with the forward LU factors: T dX^T = r^T (forward, then back substitution)
  const z64 *dX = w->Rt;
  if (!mixed) {
    CK(lu_build_perm(lb, w->perm, st));
    lb.perm = w->perm;
    CK(lu_fwdsolve_ws<z64>(T, lb, w->Rt, per, (int)N, (int)R, w->wk, st));
    CK(lu_backsolve<z64>(T, lb, w->Rt, per, (int)N, (int)R, st));
  } else {
    std::vector<char> skipm(2 * np, 0);
    for (int p : skip) skipm[2 * p] = skipm[2 * p + 1] = 1;
    int rs = tan_solve_mixed(h, (z32 *)Tv, lb, chi0q, np, w->Rt, w->Xc, skipm);
    if (rs) return rs;
    dX = w->Xc;
  }
  // dgamma^q_d
  CK(launch_gamq_tan(c, np, chi0q, dchi0q, h->c0inv, h->Frow_d, t->loc_has ? t->Fd : nullptr, w->gq, st));
  // chi sums and m_tot are bilinear: (a) with the tangents of X, gamma^w, gamma^q
  // against chi0^q and u; (b) with X, gamma^w, gamma^q against dchi0^q and du
  const z64 *gdw = t->loc_has ? t->gd : w->zero_gam, *gmw = t->loc_has ? t->gm : w->zero_gam;
  CK(launch_post(c, np, dX, 2 * per, per, (int)N, gdw, gmw, gdw, gmw, w->gq, chi0q, h->c0w, w->cA_d, w->cA_m,
                 do_eom ? w->mA : nullptr, w->eta_d, w->eta_m, h->qidx_d, st));
  DevCtx cu = c;
  cu.u = t->du;
  cu.ut = t->dut;
  cu.vq = nullptr;
  CK(launch_post(cu, np, Xp, 2 * per, per, (int)N, h->opg_d, h->opg_m, h->gam_d, h->gam_m, h->gq,
                 dchi0q ? dchi0q : w->zero_chi0, w->zero_N, w->cB_d, w->cB_m, do_eom ? w->mB : nullptr, w->eta_d,
                 w->eta_m, h->qidx_d, st));
  if (do_chi) {
    const size_t nc = (size_t)np * h->nd4;
    CK(launch_zadd(nc, w->cB_d, w->cA_d, st));
    CK(launch_zadd(nc, w->cB_m, w->cA_m, st));
    CK(cudaMemcpyAsync(t->chi_qw_d + (size_t)off * h->nd4, w->cA_d, nc * sizeof(z64), cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(t->chi_qw_m + (size_t)off * h->nd4, w->cA_m, nc * sizeof(z64), cudaMemcpyDeviceToDevice, st));
  }
  if (do_eom) {
    // dSigma += dm_tot G(k-q) + m_tot dG(k-q)
    CK(launch_zadd((size_t)np * c.nd2 * c.iwf * c.nd2, w->mB, w->mA, st));
    for (int p : skip)     // re-solved in FP64 with their tangents (m_tot of these points is zero already)
      CK(cudaMemsetAsync(w->mA + (size_t)p * c.nd2 * c.iwf * c.nd2, 0, sizeof(z64) * c.nd2 * c.iwf * c.nd2, st));
    CK(launch_eom_dynamic(c, iwb, h->qidx_d, np, w->mA, t->sigma_nl, st));
    if (t->has_dhk) {
      DevCtx cg = c;
      cg.gtab = t->gdot;
      cg.dft.ghat = t->ghat_dot;
      CK(launch_eom_dynamic(cg, iwb, h->qidx_d, np, h->mtot, t->sigma_nl, st));
    }
  }
  return 0;
}

// local tangents of direction d at omega = iwb where the block holds iq = 1
static int tan_local_update(adga_handle *h, int d, int iwb, bool do_chi, bool do_eom) {
  TanState *t = h->tan[d];
  TanWork *w = h->tw;
  DevCtx &c = h->c;
  const int wi = iwb + c.iwb;
  if (do_chi && t->loc_has)
    CK(launch_chi_loc_update(c, t->gd, t->gm, h->c0w, w->zero_nd4, t->chi_loc_d + (size_t)wi * h->nd4,
                             t->chi_loc_m + (size_t)wi * h->nd4, w->bub_scr, h->st));
  if (do_eom) {
    DevCtx cu = c;
    cu.u = t->du;
    cu.ut = t->dut;
    if (iwb == 0) CK(launch_eom_static(cu, t->sigma_dmft, h->st));
    CK(launch_eom_dmft(cu, iwb, h->gam_d, t->sigma_dmft, h->st));
    if (t->loc_has) CK(launch_eom_dmft(c, iwb, t->gd, t->sigma_dmft, h->st));
  }
  return 0;
}

// per-point outputs (and their tangents) of slot src copied to slot dst
static int move_point_outputs(adga_handle *h, int src, int dst, z64 *chi_d, z64 *chi_m, z64 *bub, bool do_chi) {
  const size_t n = h->nd4, b = sizeof(z64) * n;
  cudaStream_t st = h->st;
  CK(cudaMemcpyAsync(chi_d + dst * n, chi_d + src * n, b, cudaMemcpyDeviceToDevice, st));
  CK(cudaMemcpyAsync(chi_m + dst * n, chi_m + src * n, b, cudaMemcpyDeviceToDevice, st));
  if (bub) CK(cudaMemcpyAsync(bub + dst * n, bub + src * n, b, cudaMemcpyDeviceToDevice, st));
  if (h->tan_on && do_chi)      // tangent per-point outputs exist only with do_chi (bubble: with dH)
    for (TanState *t : h->tan)
      if (t) {
        CK(cudaMemcpyAsync(t->chi_qw_d + dst * n, t->chi_qw_d + src * n, b, cudaMemcpyDeviceToDevice, st));
        CK(cudaMemcpyAsync(t->chi_qw_m + dst * n, t->chi_qw_m + src * n, b, cudaMemcpyDeviceToDevice, st));
        if (t->has_dhk)
          CK(cudaMemcpyAsync(t->bub_nl + dst * n, t->bub_nl + src * n, b, cudaMemcpyDeviceToDevice, st));
      }
  return 0;
}

static int run_batch(adga_handle *h, int iwb, int np, int off, int prec, int *status,
                     z64 *chi_qw_d, z64 *chi_qw_m, z64 *bub_nl, bool do_eom, bool do_chi) {
  DevCtx &c = h->c;
  cudaStream_t st = h->st;
  const size_t N = c.N, R = c.R;
  const int NB = prec == ADGA_FP64 ? 64 : h->NB;
  cudaEvent_t ev[6];
  for (int i = 0; i < 6; ++i) cudaEventCreate(&ev[i]);
  CK(cudaMemcpyAsync(h->qidx_d, h->qidx_h, sizeof(int) * np, cudaMemcpyHostToDevice, st));
  cudaEventRecord(ev[0], st);
  CK(launch_chi0(c, iwb, h->qidx_d, np, h->chi0_all, h->nnu_all, st));
  z64 *chi0q = h->bigbox ? h->chi0q_big : h->chi0_all;
  CK(launch_chi0_finish(c, h->chi0_all, h->nnu_all, np, h->bubtmp, h->bigbox ? chi0q : nullptr,
                        do_chi ? bub_nl + (size_t)off * h->nd4 : nullptr, st));
  cudaEventRecord(ev[1], st);
  const size_t strideM = N * (N + R);
  LUBatch lb{(int)N, (int)(N + R), 2 * np, NB, strideM, h->ipiv, h->info, h->Linv, h->Uinv, h->rmap};
  CK(cudaMemsetAsync(h->info, 0, sizeof(int) * 2 * np, st));
  const z64 *X = nullptr;
  size_t sp = 0, sc = 0;
  int mixed_fail = 0, iters = 0;
  double worst = 0.0;
  std::vector<int> fallback;
  const int nst = (int)((N + NB - 1) / NB);
  std::vector<cudaEvent_t> tev(2 * nst);
  for (auto &x : tev) cudaEventCreate(&x);
  TrailTiming tt;
  tt.ev = tev.data();
  if (prec == ADGA_FP64) {
    z64 *T = (z64 *)h->Tm;
    CK(launch_bse_build<z64>(c, np, chi0q, h->c0inv, h->Frow_d, h->Frow_m, h->opg_d, h->opg_m, T,
                             strideM, h->gq, h->qidx_d, st));
    cudaEventRecord(ev[2], st);
    // tangents solve with L as well: keep the interchanges on the left columns
    CK(factor_batch<z64>(h, T, lb, h->tan_on, false, &tt));
    CK(lu_backsolve<z64>(T, lb, T + N * N, strideM, (int)N, (int)R, st));
    X = T + N * N; sp = 2 * strideM; sc = strideM;
  } else {
    z32 *T = (z32 *)h->Tm;
    if (h->f32_iwb != iwb) {
      CK(launch_to32(N * N, h->Frow_m, h->Frow32_m, st));
      h->f32_iwb = iwb;
    }
    CK(launch_bse_build<z32>(c, np, chi0q, h->c0inv, h->Frow_d, h->Frow_m, h->opg_d, h->opg_m, T,
                             strideM, h->gq, h->qidx_d, st, h->Frow32_m));
    cudaEventRecord(ev[2], st);
    CK(factor_batch<z32>(h, T, lb, true, h->tc != nullptr, &tt, h->mixed_nopiv));
    // the solves of the FP32 factors on the tensor cores (tune.trsv_tc = 0: streaming solves)
    lb.nopiv = h->mixed_nopiv;
    lb.tc_err = h->tune.trsv_tc ? tc_err_flag(h->tc) : nullptr;
    CK(lu_backsolve<z32>(T, lb, T + N * N, strideM, (int)N, (int)R, st));
    CK(launch_init_x(T, strideM, (int)N, (int)R, 2 * np, h->X64, st));
    CK(lu_build_perm(lb, h->perm, st));
    lb.perm = h->perm;
    const int nmat = 2 * np;
    const size_t per = N * R;
    std::vector<unsigned long long> nh(3 * nmat);
    std::vector<char> conv(nmat, 0);
    std::vector<double> rho(nmat, 1.0), xmax(nmat, 0.0);
    unsigned long long *rnorm = h->norms + 4 * (size_t)h->cap;
    auto bits = [](unsigned long long u) { double d; memcpy(&d, &u, 8); return d; };
    for (int it = 0; it < h->max_iter; ++it) {
      CK(cudaMemsetAsync(h->norms, 0, sizeof(unsigned long long) * 2 * nmat, st));
      CK(cudaMemsetAsync(rnorm, 0, sizeof(unsigned long long) * nmat, st));
      z64 *extra = nullptr;
      if (c.vq) {     // density-channel V(q) term of the residual
        const size_t ne = (size_t)np * c.nd2 * c.N;
        if (h->vq_extra_cap < ne) {
          if (h->vq_extra) cudaFree(h->vq_extra);
          h->vq_extra = nullptr;
          h->vq_extra_cap = 0;
          if (cudaMalloc(&h->vq_extra, ne * sizeof(z64)) != cudaSuccess)
            return fail(h, ADGA_ENOMEM, "V(q) residual buffer");
          h->vq_extra_cap = ne;
        }
        extra = h->vq_extra;
        CK(launch_vq_resid_extra(c, np, h->qidx_d, h->X64, chi0q, h->opg_d, extra, st));
      }
      CK(launch_residual(c, np, h->X64, chi0q, h->c0inv, h->Frow_d, h->Frow_m, h->opg_d, h->opg_m,
                         h->XD, h->V32, extra, rnorm, st, nullptr, h->tune.resid ? h->ri8 : nullptr,
                         h->frow_gen));
      if (it > 0 && h->refine_estimate) {
        // after a correction: its successor d = r A^-1 is bounded by kEstSafety * rho * max|r|,
        // rho = max|d_1| / max|r_1| of the first sweep (the solve's amplification, at least 1);
        // when that bound is within tol for every matrix the last solve is skipped
        CK(cudaMemcpyAsync(nh.data() + 2 * nmat, rnorm, sizeof(unsigned long long) * nmat,
                           cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        bool all = true;
        double west = 0.0;
        for (int m = 0; m < nmat && all; ++m) {
          const double est = kEstSafety * std::max(rho[m], 1.0) * bits(nh[2 * nmat + m]);
          const double rel = xmax[m] > 0 ? est / xmax[m] : est;
          if (!(rel <= h->tol)) all = false;
          if (!(rel <= west)) west = rel;
        }
        if (all) {
          iters = it + 1;
          worst = west;
          std::fill(conv.begin(), conv.end(), 1);
          break;
        }
      }
      CK(lu_fwdsolve_ws<z32>(T, lb, h->V32, per, (int)N, (int)R, h->work32, st));
      CK(lu_backsolve<z32>(T, lb, h->V32, per, (int)N, (int)R, st));
      CK(launch_update((int)per, nmat, h->V32, h->X64, h->norms, nullptr, st));
      CK(cudaMemcpyAsync(nh.data(), h->norms, sizeof(unsigned long long) * 2 * nmat,
                         cudaMemcpyDeviceToHost, st));
      if (it == 0)
        CK(cudaMemcpyAsync(nh.data() + 2 * nmat, rnorm, sizeof(unsigned long long) * nmat,
                           cudaMemcpyDeviceToHost, st));
      CK(cudaStreamSynchronize(st));
      iters = it + 1;
      bool all = true;
      worst = 0.0;
      for (int m = 0; m < nmat; ++m) {
        const double md = bits(nh[2 * m]), mx = bits(nh[2 * m + 1]);
        double rel = mx > 0 ? md / mx : md;
        if (!(rel <= h->tol)) all = false;
        conv[m] = rel <= h->tol;
        if (!(rel <= worst)) worst = rel;
        xmax[m] = mx;
        if (it == 0) {
          const double r1 = bits(nh[2 * nmat + m]);
          rho[m] = r1 > 0 ? md / r1 : 1.0;
        }
      }
      if (all) break;
    }
    for (int p = 0; p < np; ++p)
      if (!conv[2 * p] || !conv[2 * p + 1]) fallback.push_back(p);
    mixed_fail = (int)fallback.size();
    X = h->X64; sp = 2 * per; sc = per;
  }
  cudaEventRecord(ev[3], st);
  CK(launch_post(c, np, X, sp, sc, (int)N, h->opg_d, h->opg_m, h->gam_d, h->gam_m, h->gq, chi0q,
                 h->c0w, chi_qw_d + (size_t)off * h->nd4, chi_qw_m + (size_t)off * h->nd4,
                 do_eom ? h->mtot : nullptr, h->etad, h->etam, h->qidx_d, st));
  for (int p : fallback)    // their EOM contribution comes from the FP64 re-solve below
    CK(cudaMemsetAsync(h->mtot + (size_t)p * c.nd2 * c.iwf * c.nd2, 0,
                       sizeof(z64) * c.nd2 * c.iwf * c.nd2, st));
  cudaEventRecord(ev[4], st);
  if (do_eom) CK(launch_eom_dynamic(c, iwb, h->qidx_d, np, h->mtot, h->sigma_nl, st));
  if (h->tan_on)
    for (int d = 0; d < ADGA_MAX_TANGENTS; ++d)
      if (h->tan[d]) {
        int rt = tan_batch(h, d, iwb, np, off, h->Tm, lb, chi0q, do_chi, do_eom, prec == ADGA_MIXED, fallback);
        if (rt) return rt;
      }
  cudaEventRecord(ev[5], st);
  std::vector<int> info(2 * np);
  CK(cudaMemcpyAsync(info.data(), h->info, sizeof(int) * 2 * np, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  if (prec == ADGA_MIXED && h->tc && tc_trail_error(h->tc))
    return fail(h, ADGA_ETIMEOUT, "tensor-core trailing update: a bounded wait gave up");
  if (prec == ADGA_MIXED && h->ri8 && ri8_error(h->ri8))
    return fail(h, ADGA_ETIMEOUT, "int8-slice residual: a bounded wait gave up");
  stage_ms(h, &h->stats.ms_chi0, ev[0], ev[1]);
  stage_ms(h, &h->stats.ms_bse, ev[1], ev[2]);
  stage_ms(h, &h->stats.ms_lu, ev[2], ev[3]);
  stage_ms(h, &h->stats.ms_post, ev[3], ev[4]);
  stage_ms(h, &h->stats.ms_eom, ev[4], ev[5]);
  for (int i = 0; i < 6; ++i) cudaEventDestroy(ev[i]);
  for (int i = 0; i < tt.n; ++i) stage_ms(h, &h->stats.ms_trail, tev[2 * i], tev[2 * i + 1]);
  h->stats.trail_launches += tt.n;
  h->stats.trail_gflop += tt.gflop;
  h->stats.trail_gbytes += tt.gbytes;
  for (auto &x : tev) cudaEventDestroy(x);
  for (int p = 0; p < np; ++p) {
    int a = info[2 * p], b = info[2 * p + 1];
    int s = a ? a : b;
    if (s) h->stats.lu_info_nonzero++;
    if (status) status[off + p] = s;
  }
  h->stats.points += np;
  if (prec == ADGA_MIXED) {
    h->stats.max_refine_iters = std::max(h->stats.max_refine_iters, iters);
    if (!(worst <= h->stats.max_refine_resid)) h->stats.max_refine_resid = worst;
  }
  if (mixed_fail) {
    // FP64 re-solve of the points whose refinement did not converge, as batches:
    // their per-point outputs (and tangents) go to the scratch slots from
    // h->fb_base on, then move to their own slots.  status: -1 (re-solved), or
    // the FP64 LU's LAPACK-style info where it met an exactly zero pivot.
    std::vector<int> q(np);
    for (int p = 0; p < np; ++p) q[p] = h->qidx_h[p];
    const int mixed_cap = h->cap;
    h->stats.mixed_fallbacks += mixed_fail;
    const int saved_points = h->stats.points;
    const int base = h->fb_base;
    for (size_t f0 = 0; f0 < fallback.size();) {
      const int left = (int)(fallback.size() - f0);
      int r = ensure_work(h, ADGA_FP64, left);
      if (r) return r;
      const int nb = std::min(h->cap, left);
      for (int i = 0; i < nb; ++i) h->qidx_h[i] = q[fallback[f0 + i]];
      std::vector<int> st64((size_t)base + nb, 0);
      r = run_batch(h, iwb, nb, base, ADGA_FP64, st64.data(), chi_qw_d, chi_qw_m, bub_nl, do_eom, do_chi);
      if (r) return r;
      for (int i = 0; i < nb; ++i) {
        const int slot = off + fallback[f0 + i];
        r = move_point_outputs(h, base + i, slot, chi_qw_d, chi_qw_m, do_chi ? bub_nl : nullptr, do_chi);
        if (r) return r;
        if (status) status[slot] = st64[base + i] > 0 ? st64[base + i] : -1;
      }
      f0 += nb;
    }
    h->stats.points = saved_points;
    int r = ensure_work(h, ADGA_MIXED, mixed_cap);
    if (r) return r;
  }
  return 0;
}

// outputs of a run with npts points: the points plus as many scratch slots as a
// batch can hold (the FP64 re-solve of unconverged mixed points writes there)
static int out_slots(const adga_handle *h, int npts) { return npts + std::min(npts, h->c.nqp); }

static void free_owned(adga_handle *h, void *p) {
  if (!p) return;
  auto it = std::find(h->owned.begin(), h->owned.end(), p);
  if (it != h->owned.end()) h->owned.erase(it);
  cudaFree(p);
}

static int ensure_outputs(adga_handle *h, int npts) {
  const int want = out_slots(h, npts);
  if (h->out_cap >= want) return 0;
  // superseded buffers of earlier (smaller) runs are freed
  cudaStreamSynchronize(h->st);
  free_owned(h, h->chi_qw_d);
  free_owned(h, h->chi_qw_m);
  free_owned(h, h->bubble_nl);
  h->chi_qw_d = h->chi_qw_m = h->bubble_nl = nullptr;
  h->out_cap = 0;
  auto &L = h->owned;
  if (!alloc_into(h, h->chi_qw_d, (size_t)want * h->nd4, L) ||
      !alloc_into(h, h->chi_qw_m, (size_t)want * h->nd4, L) ||
      !alloc_into(h, h->bubble_nl, (size_t)want * h->nd4, L))
    return fail(h, ADGA_ENOMEM, "per-point outputs");
  h->out_cap = want;
  return 0;
}

extern "C" int adga_ladder_run(adga_handle *h, int qwstart, int qwstop, int precision, int *status,
                               adga_run_stats *stats) {
  if (!h) return ADGA_EINVAL;
  DevCtx &c = h->c;
  const int total = c.nqp * h->nw;
  if (qwstart < 1 || qwstop > total || qwstop < qwstart)
    return fail(h, ADGA_EINVAL, "qw range outside 1..nqp*(2*iwbmax_small+1)");
  if (precision != ADGA_FP64 && precision != ADGA_MIXED) return fail(h, ADGA_EINVAL, "precision");
  // the tuned mixed path may factor in FP64 (tune.factor = 1: faster at this size)
  if (precision == ADGA_MIXED && h->tune.factor == 1) precision = ADGA_FP64;
  const int npts = qwstop - qwstart + 1;
  int r = ensure_outputs(h, npts);
  if (r) return r;
  h->fb_base = npts;
  memset(&h->stats, 0, sizeof(h->stats));
  const long long launches0 = g_adga_launches.load();
  CK(cudaMemsetAsync(h->chi_qw_d, 0, sizeof(z64) * npts * h->nd4, h->st));
  CK(cudaMemsetAsync(h->chi_qw_m, 0, sizeof(z64) * npts * h->nd4, h->st));
  CK(cudaMemsetAsync(h->bubble_nl, 0, sizeof(z64) * npts * h->nd4, h->st));
  r = ensure_work(h, precision, std::min(npts, c.nqp));
  if (r) return r;
  cudaEventRecord(h->e0, h->st);
  const bool do_chi = h->d.do_chi != 0, do_eom = h->d.do_eom != 0;
  int p = 0;
  while (p < npts) {
    const int qw = qwstart + p;               // 1-based compound index
    const int iwb = -c.iwb + (qw - 1) / c.nqp;
    const int iq0 = (qw - 1) % c.nqp;
    const int seg = std::min(npts - p, c.nqp - iq0);
    r = ensure_local(h, iwb);
    if (r) return r;
    for (int d = 0; h->tan_on && d < ADGA_MAX_TANGENTS; ++d)
      if (h->tan[d] && (r = tan_local(h, d, iwb))) return r;
    if (iq0 == 0) {
      for (int d = 0; h->tan_on && d < ADGA_MAX_TANGENTS; ++d)
        if (h->tan[d] && (r = tan_local_update(h, d, iwb, do_chi, do_eom))) return r;
      if (do_chi)
        CK(launch_chi_loc_update(c, h->gam_d, h->gam_m, h->c0w, h->bubtmp,
                                 h->ext_cld ? nullptr : h->chi_loc_d + (size_t)(iwb + c.iwb) * h->nd4,
                                 h->ext_cld ? nullptr : h->chi_loc_m + (size_t)(iwb + c.iwb) * h->nd4,
                                 h->bubble_loc + (size_t)(iwb + c.iwb) * h->nd4, h->st));
      if (do_eom) {
        if (iwb == 0) CK(launch_eom_static(c, h->sigma_dmft, h->st));
        CK(launch_eom_dmft(c, iwb, h->gam_d, h->sigma_dmft, h->st));
      }
    }
    for (int b0 = 0; b0 < seg; b0 += h->cap) {
      const int nb = std::min(h->cap, seg - b0);
      for (int i = 0; i < nb; ++i) h->qidx_h[i] = iq0 + b0 + i;
      if (do_eom && iwb == 0 && c.vq) {   // calc_eom_static's V(q) terms, every q (src/main.F90:635-637)
        CK(cudaMemcpyAsync(h->qidx_d, h->qidx_h, sizeof(int) * nb, cudaMemcpyHostToDevice, h->st));
        CK(launch_eom_static_vq(c, h->qidx_d, nb, h->sigma_hf, h->st));
      }
      r = run_batch(h, iwb, nb, p + b0, precision, status, h->chi_qw_d, h->chi_qw_m, h->bubble_nl,
                    do_eom, do_chi);
      if (r) return r;
    }
    p += seg;
  }
  cudaEventRecord(h->e1, h->st);
  CK(cudaStreamSynchronize(h->st));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, h->e0, h->e1);
  h->stats.ms_total = ms;
  h->stats.kernel_launches = g_adga_launches.load() - launches0;
  h->last_npts = npts;
  if (stats) *stats = h->stats;
  return 0;
}

// ---------------------------------------------------------------------------
// kernel choices of the mixed path and the autotuner
// ---------------------------------------------------------------------------
extern "C" int adga_set_tune(adga_handle *h, const adga_tune *t) {
  if (!h || !t) return ADGA_EINVAL;
  if (t->factor < 0 || t->factor > 1 || t->pairs < 0 || t->pairs > 3 || t->tri_tc < 0 || t->tri_tc > 1 ||
      t->batch < 0 || t->resid < 0 || t->resid > 1 || t->trsv_tc < 0 || t->trsv_tc > 1)
    return fail(h, ADGA_EINVAL,
                "adga_set_tune: factor, tri_tc, resid, trsv_tc in {0, 1}, pairs in {0, 1, 2, 3}, batch >= 0");
  h->tune = *t;
  return 0;
}

extern "C" int adga_get_tune(const adga_handle *h, adga_tune *t) {
  if (!h || !t) return ADGA_EINVAL;
  *t = h->tune;
  return 0;
}

// one run of qwstart..qwstop from zeroed accumulators; host copies of the
// per-point chi and of Sigma_nl
static int tune_sample(adga_handle *h, int qwstart, int qwstop, int prec, std::vector<z64> &chi,
                       std::vector<z64> &sig, double *ms) {
  int r = adga_reset_outputs(h);
  if (r) return r;
  adga_run_stats st{};
  if ((r = adga_ladder_run(h, qwstart, qwstop, prec, nullptr, &st))) return r;
  const size_t nc = (size_t)(qwstop - qwstart + 1) * h->nd4;
  const size_t ns = (size_t)h->c.nd2 * 2 * h->c.iwf * h->c.nkp_eom;
  chi.resize(2 * nc);
  sig.resize(ns);
  CK(cudaMemcpy(chi.data(), h->chi_qw_d, nc * sizeof(z64), cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(chi.data() + nc, h->chi_qw_m, nc * sizeof(z64), cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(sig.data(), h->sigma_nl, ns * sizeof(z64), cudaMemcpyDeviceToHost));
  *ms = st.ms_total;
  return 0;
}

static double rel_diff(const std::vector<z64> &a, const std::vector<z64> &b, size_t lo, size_t hi) {
  double num = 0.0, den = 0.0;
  for (size_t i = lo; i < hi; ++i) {
    const double d = std::max(std::fabs(a[i].x - b[i].x), std::fabs(a[i].y - b[i].y));
    const double m = std::max(std::fabs(b[i].x), std::fabs(b[i].y));
    if (!(d <= num)) num = d;    // NaN propagates
    den = std::max(den, m);
  }
  return den > 0 ? num / den : num;
}

extern "C" int adga_autotune(adga_handle *h, int qwstart, int qwstop, double tol, adga_tune_trial *trials,
                             int max_trials, int *ntrials, adga_tune *best) {
  if (!h) return ADGA_EINVAL;
  const DevCtx &c = h->c;
  if (qwstart < 1 || qwstop > c.nqp * h->nw || qwstop < qwstart)
    return fail(h, ADGA_EINVAL, "adga_autotune: qw range outside 1..nqp*(2*iwbmax_small+1)");
  if (h->tan_on) return fail(h, ADGA_ESTATE, "adga_autotune: not inside a tangent run");
  if (!(tol > 0)) tol = 1e-8;
  const adga_tune start = h->tune;
  // candidates: the tensor-core variants (when the tensor cores serve this size), then
  // the FP64 factorisation
  std::vector<adga_tune> cand;
  auto with = [&](int f, int p, int t, int rs, int ts) {
    adga_tune x = start; x.factor = f; x.pairs = p; x.tri_tc = t; x.resid = rs; x.trsv_tc = ts; return x;
  };
  const bool tc = tc_available() && !getenv("ADGA_NO_TC");
  if (tc) {
    if (c.N % 2 == 0) {
      cand.push_back(with(0, 2, 1, 1, 1));
      cand.push_back(with(0, 3, 1, 1, 1));
      cand.push_back(with(0, 1, 1, 1, 1));
      cand.push_back(with(0, 2, 1, 1, 0));
      cand.push_back(with(0, 2, 1, 0, 1));
    }
    cand.push_back(with(0, 1, 0, 1, 0));
    cand.push_back(with(0, 0, 0, 1, 0));
  } else {
    cand.push_back(with(0, 0, 0, 0, 0));
  }
  cand.push_back(with(1, 0, 0, 0, 0));
  std::vector<z64> ref_chi, ref_sig, chi, sig;
  double ms = 0.0;
  h->tune = start;
  int r = tune_sample(h, qwstart, qwstop, ADGA_FP64, ref_chi, ref_sig, &ms);
  const size_t nc = ref_chi.size() / 2;
  int nt = 0, ibest = -1;
  double best_ms = 0.0;
  for (size_t i = 0; !r && i < cand.size(); ++i) {
    h->tune = cand[i];
    double ms_warm = 0.0;
    if ((r = tune_sample(h, qwstart, qwstop, ADGA_MIXED, chi, sig, &ms_warm))) break;
    if ((r = tune_sample(h, qwstart, qwstop, ADGA_MIXED, chi, sig, &ms))) break;
    const double err = std::max({rel_diff(chi, ref_chi, 0, nc), rel_diff(chi, ref_chi, nc, 2 * nc),
                                 rel_diff(sig, ref_sig, 0, sig.size())});
    const bool ok = err <= tol;
    if (trials && nt < max_trials) trials[nt] = adga_tune_trial{cand[i], ms, err, ok ? 1 : 0};
    ++nt;
    if (ok && (ibest < 0 || ms < best_ms)) { ibest = (int)i; best_ms = ms; }
  }
  h->tune = (!r && ibest >= 0) ? cand[ibest] : start;
  if (ntrials) *ntrials = nt;
  if (best) *best = h->tune;
  int r2 = adga_reset_outputs(h);
  return r ? r : r2;
}

extern "C" int adga_ladder_run_tangent(adga_handle *h, int qwstart, int qwstop, int precision, int *status,
                                       adga_run_stats *stats) {
  if (!h) return ADGA_EINVAL;
  int ndir = 0;
  for (TanState *t : h->tan) ndir += t != nullptr;
  if (!ndir) return fail(h, ADGA_ESTATE, "ladder_run_tangent: no tangent direction set");
  if (h->c.vq) return fail(h, ADGA_EINVAL, "ladder_run_tangent: V(q) tangents are not supported");
  const DevCtx &c = h->c;
  if (qwstart < 1 || qwstop > c.nqp * h->nw || qwstop < qwstart) return fail(h, ADGA_EINVAL, "qw range");
  const int npts = qwstop - qwstart + 1;
  for (TanState *t : h->tan) {
    if (!t) continue;
    const int want = out_slots(h, npts);
    if (t->out_cap < want) {
      cudaStreamSynchronize(h->st);
      for (z64 *p : {t->chi_qw_d, t->chi_qw_m, t->bub_nl}) if (p) cudaFree(p);
      t->chi_qw_d = t->chi_qw_m = t->bub_nl = nullptr;
      t->out_cap = 0;
      if (cudaMalloc(&t->chi_qw_d, sizeof(z64) * want * h->nd4) != cudaSuccess ||
          cudaMalloc(&t->chi_qw_m, sizeof(z64) * want * h->nd4) != cudaSuccess ||
          cudaMalloc(&t->bub_nl, sizeof(z64) * want * h->nd4) != cudaSuccess)
        return fail(h, ADGA_ENOMEM, "tangent per-point outputs");
      t->out_cap = want;
    }
    CK(cudaMemsetAsync(t->chi_qw_d, 0, sizeof(z64) * npts * h->nd4, h->st));
    CK(cudaMemsetAsync(t->chi_qw_m, 0, sizeof(z64) * npts * h->nd4, h->st));
    CK(cudaMemsetAsync(t->bub_nl, 0, sizeof(z64) * npts * h->nd4, h->st));
    t->loc_iwb = INT_MIN;
  }
  h->tan_on = true;
  h->loc_iwb = INT_MIN;
  if (precision != ADGA_FP64 && precision != ADGA_MIXED) return fail(h, ADGA_EINVAL, "precision");
  int r = adga_ladder_run(h, qwstart, qwstop, precision, status, stats);
  h->tan_on = false;
  return r;
}

extern "C" int adga_get_tangent_outputs(adga_handle *h, int dir, const adga_outputs *o) {
  if (!h || !o) return ADGA_EINVAL;
  if (!tan_dir_ok(dir) || !h->tan[dir]) return fail(h, ADGA_ESTATE, "get_tangent_outputs: direction not set");
  TanState *t = h->tan[dir];
  const DevCtx &c = h->c;
  cudaStream_t st = h->st;
  CK(launch_mirror_sigma(c, t->sigma_nl, c.nkp_eom, st));
  const size_t np = h->last_npts;
#define TDN(dst, src, n) \
  if (dst) CK(cudaMemcpyAsync(dst, src, sizeof(z64) * (n), cudaMemcpyDeviceToHost, st))
  if (np && t->chi_qw_d) {
    TDN(o->chi_qw_dens, t->chi_qw_d, np * h->nd4);
    TDN(o->chi_qw_magn, t->chi_qw_m, np * h->nd4);
    TDN(o->bubble_nl, t->bub_nl, np * h->nd4);
  }
  TDN(o->chi_loc_dens, t->chi_loc_d, (size_t)h->nd4 * h->nw);
  TDN(o->chi_loc_magn, t->chi_loc_m, (size_t)h->nd4 * h->nw);
  TDN(o->sigma_nl, t->sigma_nl, (size_t)c.nd2 * 2 * c.iwf * c.nkp_eom);
  TDN(o->sigma_dmft, t->sigma_dmft, (size_t)c.nd2 * 2 * c.iwf);
#undef TDN
  CK(cudaStreamSynchronize(st));
  // the local bubble and sigma_hf do not depend on the direction (G_loc, n fixed; no V(q))
  if (o->bubble_loc) memset(o->bubble_loc, 0, sizeof(z64) * h->nd4 * h->nw);
  if (o->sigma_hf) memset(o->sigma_hf, 0, sizeof(z64) * c.nd2 * c.nkp_eom);
  return 0;
}

extern "C" int adga_post_loop(adga_handle *h, adga_z *sigma_sum, adga_z *sigma_loc, adga_z *gloc,
                              adga_z *n_dga_k, adga_z *n_dga) {
  if (!h) return ADGA_EINVAL;
  const DevCtx &c = h->c;
  cudaStream_t st = h->st;
  const bool full_mesh = c.nkp_eom == c.nkp && !c.keom;
  if ((sigma_loc || gloc) && !full_mesh)
    return fail(h, ADGA_EINVAL, "post_loop: sigma_loc / gloc need the EOM on the full k mesh");
  if (c.nd > GINV_MAXND_HOST) return fail(h, ADGA_EINVAL, "post_loop: ndim above 8");
  const size_t ns = (size_t)c.nd2 * 2 * c.iwf * c.nkp_eom, ngl = (size_t)2 * c.iwmax * c.nd2;
  const size_t nsl = (size_t)c.nd2 * 2 * c.iwf, nnk = (size_t)c.nkp_eom * c.nd2;
  z64 *buf = nullptr;
  const size_t total = ns + nsl + ngl + nnk + c.nd;
  if (cudaMalloc(&buf, total * sizeof(z64)) != cudaSuccess) return fail(h, ADGA_ENOMEM, "post_loop buffers");
  z64 *sig = buf, *sl = sig + ns, *gl = sl + nsl, *nk = gl + ngl, *n = nk + nnk;
  cudaError_t e;
  if (sigma_sum) {
    e = cudaMemcpyAsync(sig, sigma_sum, ns * sizeof(z64), cudaMemcpyHostToDevice, st);
  } else {
    // this handle's own non-local Sigma, mirrored (src/eom_module.f90:228)
    e = launch_mirror_sigma(c, h->sigma_nl, c.nkp_eom, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(sig, h->sigma_nl, ns * sizeof(z64), cudaMemcpyDeviceToDevice, st);
  }
  if (e == cudaSuccess)
    e = launch_post_loop(c, c.keom, sig, sigma_loc ? sl : nullptr, gloc ? gl : nullptr,
                         (n_dga_k || n_dga) ? nk : nullptr, n_dga ? n : nullptr, st);
#define PDN(dst, src, cnt) \
  if (e == cudaSuccess && dst) e = cudaMemcpyAsync(dst, src, (cnt) * sizeof(z64), cudaMemcpyDeviceToHost, st)
  PDN(sigma_sum, sig, ns);
  PDN(sigma_loc, sl, nsl);
  PDN(gloc, gl, ngl);
  PDN(n_dga_k, nk, nnk);
  PDN(n_dga, n, (size_t)c.nd);
#undef PDN
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaFree(buf);
  if (e != cudaSuccess) return fail(h, ADGA_ECUDA, std::string("post_loop: ") + cudaGetErrorString(e));
  return 0;
}

extern "C" int adga_get_outputs(adga_handle *h, const adga_outputs *o) {
  if (!h || !o) return ADGA_EINVAL;
  const DevCtx &c = h->c;
  cudaStream_t st = h->st;
  // Sigma(-nu-1) = Sigma(nu)^dagger (src/eom_module.f90:228)
  CK(launch_mirror_sigma(c, h->sigma_nl, c.nkp_eom, st));
  const size_t np = h->last_npts;
#define DN(dst, src, n) \
  if (dst) CK(cudaMemcpyAsync(dst, src, sizeof(z64) * (n), cudaMemcpyDeviceToHost, st))
  if (np) {
    DN(o->chi_qw_dens, h->chi_qw_d, np * h->nd4);
    DN(o->chi_qw_magn, h->chi_qw_m, np * h->nd4);
    DN(o->bubble_nl, h->bubble_nl, np * h->nd4);
  }
  DN(o->bubble_loc, h->bubble_loc, (size_t)h->nd4 * h->nw);
  // an external chi_loc (read_chi_loc) replaces the one built from gamma^w
  DN(o->chi_loc_dens, h->ext_cld ? h->ext_cld : h->chi_loc_d, (size_t)h->nd4 * h->nw);
  DN(o->chi_loc_magn, h->ext_clm ? h->ext_clm : h->chi_loc_m, (size_t)h->nd4 * h->nw);
  DN(o->sigma_nl, h->sigma_nl, (size_t)c.nd2 * 2 * c.iwf * c.nkp_eom);
  DN(o->sigma_dmft, h->sigma_dmft, (size_t)c.nd2 * 2 * c.iwf);
  DN(o->sigma_hf, h->sigma_hf, (size_t)c.nd2 * c.nkp_eom);
#undef DN
  CK(cudaStreamSynchronize(st));
  return 0;
}

// ---------------------------------------------------------------------------
// per-routine entry points
// ---------------------------------------------------------------------------
extern "C" int adga_get_chi0_loc(adga_handle *h, int iwf, int iwb, adga_z *out) {
  if (!h || !out) return ADGA_EINVAL;
  const DevCtx &c = h->c;
  if (iwf < -c.iwf || iwf >= c.iwf || iwb < -c.iwb || iwb > c.iwb) return ADGA_EINVAL;
  int r = ensure_diag(h, iwb);
  if (r) return r;
  std::vector<z64> d(c.nd2);
  CK(cudaMemcpyAsync(d.data(), h->c0w + (size_t)(iwf + c.iwf) * c.nd2, sizeof(z64) * c.nd2,
                     cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  memset(out, 0, sizeof(adga_z) * c.nd2 * c.nd2);
  for (int i = 0; i < c.nd2; ++i) memcpy(&out[i + i * c.nd2], &d[i], sizeof(adga_z));
  return 0;
}

extern "C" int adga_get_chi0_loc_inv(adga_handle *h, int iwf, int iwb, adga_z *out) {
  if (!h || !out) return ADGA_EINVAL;
  const DevCtx &c = h->c;
  if (iwf < -c.iwf || iwf >= c.iwf || iwb < -c.iwb || iwb > c.iwb) return ADGA_EINVAL;
  int r = ensure_diag(h, iwb);
  if (r) return r;
  std::vector<z64> d(c.nd2);
  CK(cudaMemcpyAsync(d.data(), h->c0inv + (size_t)(iwf + c.iwf) * c.nd2, sizeof(z64) * c.nd2,
                     cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  memset(out, 0, sizeof(adga_z) * c.nd2 * c.nd2);
  for (int i = 0; i < c.nd2; ++i) memcpy(&out[i + i * c.nd2], &d[i], sizeof(adga_z));
  return 0;
}

extern "C" int adga_chi0_q(adga_handle *h, int iq, int iwb, adga_z *chi0q, adga_z *bubble_nl) {
  if (!h) return ADGA_EINVAL;
  DevCtx &c = h->c;
  if (iq < 1 || iq > c.nqp || iwb < -c.iwb || iwb > c.iwb) return ADGA_EINVAL;
  int r = ensure_diag(h, iwb);
  if (r) return r;
  const int prec = h->cap_prec < 0 ? ADGA_FP64 : h->cap_prec;
  r = ensure_work(h, prec, 1);
  if (r) return r;
  h->qidx_h[0] = iq - 1;
  CK(cudaMemcpyAsync(h->qidx_d, h->qidx_h, sizeof(int), cudaMemcpyHostToDevice, h->st));
  CK(launch_chi0(c, iwb, h->qidx_d, 1, h->chi0_all, h->nnu_all, h->st));
  z64 *bn = h->etad;   // scratch
  CK(launch_chi0_finish(c, h->chi0_all, h->nnu_all, 1, h->bubtmp, h->bigbox ? h->chi0q_big : nullptr,
                        bn, h->st));
  const z64 *src = h->bigbox ? h->chi0q_big : h->chi0_all;
  if (chi0q)
    CK(cudaMemcpyAsync(chi0q, src, sizeof(z64) * h->nd4 * 2 * c.iwf, cudaMemcpyDeviceToHost, h->st));
  if (bubble_nl)
    CK(cudaMemcpyAsync(bubble_nl, bn, sizeof(z64) * h->nd4, cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  return 0;
}

extern "C" int adga_get_gamma_w(adga_handle *h, int iwb, adga_z *gd, adga_z *gm) {
  if (!h) return ADGA_EINVAL;
  if (iwb < -h->c.iwb || iwb > h->c.iwb) return ADGA_EINVAL;
  int r = ensure_local(h, iwb);
  if (r) return r;
  const size_t n = (size_t)h->c.nd2 * h->c.N;
  if (gd) CK(cudaMemcpyAsync(gd, h->gam_d, sizeof(z64) * n, cudaMemcpyDeviceToHost, h->st));
  if (gm) CK(cudaMemcpyAsync(gm, h->gam_m, sizeof(z64) * n, cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  return 0;
}

extern "C" int adga_bse_point(adga_handle *h, int iq, int iwb, int precision, adga_z *etaqd,
                              adga_z *etaqm, adga_z *gammaqd, int *lu_info) {
  if (!h) return ADGA_EINVAL;
  DevCtx &c = h->c;
  if (iq < 1 || iq > c.nqp || iwb < -c.iwb || iwb > c.iwb) return ADGA_EINVAL;
  if (precision != ADGA_FP64 && precision != ADGA_MIXED) return ADGA_EINVAL;
  int r = ensure_local(h, iwb);
  if (r) return r;
  r = ensure_work(h, precision, 1);
  if (r) return r;
  z64 *scr = nullptr;
  std::vector<void *> tmp;
  // per-point outputs: the point's slot and one scratch slot for a re-solve
  if (!alloc_into(h, scr, (size_t)6 * h->nd4, tmp)) return fail(h, ADGA_ENOMEM, "scratch");
  h->qidx_h[0] = iq - 1;
  int st_info[2] = {0, 0};
  memset(&h->stats, 0, sizeof(h->stats));
  h->fb_base = 1;
  r = run_batch(h, iwb, 1, 0, precision, st_info, scr, scr + 2 * h->nd4, scr + 4 * h->nd4, false, true);
  if (!r && h->stats.mixed_fallbacks) {
    // the mixed refinement did not converge: eta and gamma^q_d from the FP64 path
    r = ensure_work(h, ADGA_FP64, 1);
    if (!r) {
      h->qidx_h[0] = iq - 1;
      r = run_batch(h, iwb, 1, 0, ADGA_FP64, st_info, scr, scr + 2 * h->nd4, scr + 4 * h->nd4, false, true);
    }
  }
  if (!r) {
    const size_t n = (size_t)c.nd2 * c.N;
    if (etaqd) cudaMemcpyAsync(etaqd, h->etad, sizeof(z64) * n, cudaMemcpyDeviceToHost, h->st);
    if (etaqm) cudaMemcpyAsync(etaqm, h->etam, sizeof(z64) * n, cudaMemcpyDeviceToHost, h->st);
    if (gammaqd) cudaMemcpyAsync(gammaqd, h->gq, sizeof(z64) * n, cudaMemcpyDeviceToHost, h->st);
    if (cudaStreamSynchronize(h->st) != cudaSuccess) r = fail(h, ADGA_ECUDA, "copy-out");
  }
  free_list(tmp);
  if (lu_info) *lu_info = st_info[0];
  return r;
}

extern "C" int adga_calc_chi_qw(adga_handle *h, adga_z *chi_qw, const adga_z *interm3,
                                const adga_z *chi0_sum) {
  if (!h || !chi_qw || !interm3 || !chi0_sum) return ADGA_EINVAL;
  const DevCtx &c = h->c;
  std::vector<void *> tmp;
  z64 *dchi, *dim3_, *dc0;
  const size_t nI = (size_t)c.nd2 * c.N, nC = (size_t)h->nd4 * 2 * c.iwf;
  if (!alloc_into(h, dchi, h->nd4, tmp) || !alloc_into(h, dim3_, nI, tmp) ||
      !alloc_into(h, dc0, nC, tmp)) {
    free_list(tmp);
    return fail(h, ADGA_ENOMEM, "calc_chi_qw buffers");
  }
  cudaStream_t st = h->st;
  cudaMemcpyAsync(dchi, chi_qw, sizeof(z64) * h->nd4, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(dim3_, interm3, sizeof(z64) * nI, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(dc0, chi0_sum, sizeof(z64) * nC, cudaMemcpyHostToDevice, st);
  cudaError_t e = launch_calc_chi_qw(c, dchi, dim3_, dc0, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(chi_qw, dchi, sizeof(z64) * h->nd4, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  free_list(tmp);
  if (e != cudaSuccess) return fail(h, ADGA_ECUDA, cudaGetErrorString(e));
  return 0;
}

// m_tot from eta_d, eta_m, gamma^q_d for one point (same kernel as the batch post)
extern "C" int adga_calc_eom_dynamic(adga_handle *h, const adga_z *etaqd, const adga_z *etaqm,
                                     const adga_z *gammaqd, int iwb, int iq, adga_z *sigma_nl) {
  if (!h || !etaqd || !etaqm || !gammaqd || !sigma_nl) return ADGA_EINVAL;
  DevCtx &c = h->c;
  if (iq < 1 || iq > c.nqp || iwb < -c.iwb || iwb > c.iwb) return ADGA_EINVAL;
  const int prec = h->cap_prec < 0 ? ADGA_FP64 : h->cap_prec;
  int r = ensure_work(h, prec, 1);
  if (r) return r;
  const size_t n = (size_t)c.nd2 * c.N, ns = (size_t)c.nd2 * 2 * c.iwf * c.nkp_eom;
  std::vector<void *> tmp;
  z64 *X, *scr, *chi0z, *opz, *sig;
  if (!alloc_into(h, X, 2 * n, tmp) || !alloc_into(h, scr, 2 * h->nd4, tmp) ||
      !alloc_into(h, chi0z, (size_t)h->nd4 * 2 * c.iwf, tmp) || !alloc_into(h, opz, n, tmp) ||
      !alloc_into(h, sig, ns, tmp)) {
    free_list(tmp);
    return fail(h, ADGA_ENOMEM, "eom buffers");
  }
  cudaStream_t st = h->st;
  // Feed eta through the post kernel as X = eta^T with zero (1+gamma): it
  // rebuilds eta and forms m_tot with the reference's coefficients.
  std::vector<adga_z> xt(2 * n);
  for (int i1 = 0; i1 < c.nd2; ++i1)
    for (int cc = 0; cc < c.N; ++cc) {
      xt[cc + (size_t)i1 * c.N] = etaqd[i1 + (size_t)cc * c.nd2];
      xt[n + cc + (size_t)i1 * c.N] = etaqm[i1 + (size_t)cc * c.nd2];
    }
  cudaError_t e = cudaMemcpyAsync(X, xt.data(), sizeof(z64) * 2 * n, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(opz, 0, sizeof(z64) * n, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(chi0z, 0, sizeof(z64) * h->nd4 * 2 * c.iwf, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(h->gq, gammaqd, sizeof(z64) * n, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(sig, sigma_nl, sizeof(z64) * ns, cudaMemcpyHostToDevice, st);
  h->qidx_h[0] = iq - 1;
  if (e == cudaSuccess) e = cudaMemcpyAsync(h->qidx_d, h->qidx_h, sizeof(int), cudaMemcpyHostToDevice, st);
  // with V(q), m_tot also needs gamma^w_d of this omega (src/eom_module.f90:202-205)
  const z64 *gwd = opz;
  if (e == cudaSuccess && c.vq) {
    int rl = ensure_local(h, iwb);
    if (rl) { free_list(tmp); return rl; }
    gwd = h->gam_d;
  }
  if (e == cudaSuccess)
    e = launch_post(c, 1, X, 2 * n, n, c.N, opz, opz, gwd, opz, h->gq, chi0z, h->c0w, scr, scr + h->nd4,
                    h->mtot, h->etad, h->etam, h->qidx_d, st);
  if (e == cudaSuccess) e = launch_eom_dynamic(c, iwb, h->qidx_d, 1, h->mtot, sig, st);
  if (e == cudaSuccess) e = launch_mirror_sigma(c, sig, c.nkp_eom, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(sigma_nl, sig, sizeof(z64) * ns, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  free_list(tmp);
  if (e != cudaSuccess) return fail(h, ADGA_ECUDA, cudaGetErrorString(e));
  return 0;
}

extern "C" int adga_calc_eom_dmft(adga_handle *h, const adga_z *gammawd, int iwb, adga_z *sigma_dmft) {
  if (!h || !gammawd || !sigma_dmft) return ADGA_EINVAL;
  DevCtx &c = h->c;
  if (iwb < -c.iwb || iwb > c.iwb) return ADGA_EINVAL;
  const size_t n = (size_t)c.nd2 * c.N, ns = (size_t)c.nd2 * 2 * c.iwf;
  std::vector<void *> tmp;
  z64 *g, *s;
  if (!alloc_into(h, g, n, tmp) || !alloc_into(h, s, ns, tmp)) {
    free_list(tmp);
    return fail(h, ADGA_ENOMEM, "eom_dmft buffers");
  }
  cudaStream_t st = h->st;
  cudaError_t e = cudaMemcpyAsync(g, gammawd, sizeof(z64) * n, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(s, sigma_dmft, sizeof(z64) * ns, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = launch_eom_dmft(c, iwb, g, s, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(sigma_dmft, s, sizeof(z64) * ns, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  free_list(tmp);
  if (e != cudaSuccess) return fail(h, ADGA_ECUDA, cudaGetErrorString(e));
  return 0;
}

extern "C" int adga_calc_eom_static(adga_handle *h, int iq, adga_z *sigma_dmft) {
  if (!h || !sigma_dmft) return ADGA_EINVAL;
  if (iq != 1) return 0;       // the local Hartree term only enters at q = 1
  DevCtx &c = h->c;
  const size_t ns = (size_t)c.nd2 * 2 * c.iwf;
  std::vector<void *> tmp;
  z64 *s;
  if (!alloc_into(h, s, ns, tmp)) return fail(h, ADGA_ENOMEM, "eom_static buffers");
  cudaStream_t st = h->st;
  cudaError_t e = cudaMemcpyAsync(s, sigma_dmft, sizeof(z64) * ns, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = launch_eom_static(c, s, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(sigma_dmft, s, sizeof(z64) * ns, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  free_list(tmp);
  if (e != cudaSuccess) return fail(h, ADGA_ECUDA, cudaGetErrorString(e));
  return 0;
}

// ---------------------------------------------------------------------------
// standalone helpers
// ---------------------------------------------------------------------------
extern "C" int adga_inverse_matrix_z(adga_z *M, int n, int *ierr, char *erstr) {
  if (!M || n < 1 || n > 4096) return ADGA_EINVAL;
  const int NB = 64, nsteps = (n + NB - 1) / NB;
  const size_t strideM = (size_t)n * 2 * n;
  z64 *T = nullptr, *Li = nullptr, *Ui = nullptr;
  int *ip = nullptr, *inf = nullptr, *rm = nullptr;
  cudaStream_t st;
  if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return ADGA_ECUDA;
  int rc = 0;
  std::vector<adga_z> aug((size_t)n * 2 * n);
  memcpy(aug.data(), M, sizeof(adga_z) * n * n);
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) {
      adga_z v = {i == j ? 1.0 : 0.0, 0.0};
      aug[(size_t)n * n + i + (size_t)j * n] = v;
    }
  if (cudaMalloc(&T, sizeof(z64) * strideM) != cudaSuccess ||
      cudaMalloc(&Li, sizeof(z64) * nsteps * NB * NB) != cudaSuccess ||
      cudaMalloc(&Ui, sizeof(z64) * nsteps * NB * NB) != cudaSuccess ||
      cudaMalloc(&ip, sizeof(int) * n) != cudaSuccess || cudaMalloc(&inf, sizeof(int)) != cudaSuccess ||
      cudaMalloc(&rm, sizeof(int) * RMAP_STRIDE) != cudaSuccess) {
    rc = ADGA_ENOMEM;
  } else {
    LUBatch lb{n, 2 * n, 1, NB, strideM, ip, inf, Li, Ui, rm};
    int info = 0;
    cudaError_t e = cudaMemcpyAsync(T, aug.data(), sizeof(z64) * strideM, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(inf, 0, sizeof(int), st);
    if (e == cudaSuccess) e = lu_factor<z64>(T, lb, false, nullptr, nullptr, st);
    if (e == cudaSuccess) e = lu_backsolve<z64>(T, lb, T + (size_t)n * n, strideM, n, n, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&info, inf, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(M, T + (size_t)n * n, sizeof(z64) * n * n, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) rc = ADGA_ECUDA;
    if (ierr) *ierr = info;
    if (erstr) {
      if (info) snprintf(erstr, 200, "ERROR in ZGETRF");
      else erstr[0] = 0;
    }
    if (rc == 0 && info) rc = info;
  }
  cudaFree(T); cudaFree(Li); cudaFree(Ui); cudaFree(ip); cudaFree(inf); cudaFree(rm);
  cudaStreamDestroy(st);
  return rc;
}

extern "C" int adga_index_kq(int nkpx, int nkpy, int nkpz, const int *q_data, int nqp,
                             const int *k_sel, int nk_sel, int *ind) {
  if (!q_data || !ind || nqp < 1 || nkpx < 1 || nkpy < 1 || nkpz < 1) return ADGA_EINVAL;
  const int nkp = nkpx * nkpy * nkpz;
  const int nk = k_sel ? nk_sel : nkp;
  int *dq = nullptr, *dk = nullptr, *di = nullptr;
  int rc = 0;
  if (cudaMalloc(&dq, sizeof(int) * nqp) != cudaSuccess || cudaMalloc(&di, sizeof(int) * (size_t)nk * nqp) != cudaSuccess ||
      (k_sel && cudaMalloc(&dk, sizeof(int) * nk) != cudaSuccess)) {
    rc = ADGA_ENOMEM;
  } else {
    cudaError_t e = cudaMemcpy(dq, q_data, sizeof(int) * nqp, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && k_sel) e = cudaMemcpy(dk, k_sel, sizeof(int) * nk, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = launch_kq_index(nkpx, nkpy, nkpz, dk, nk, dq, nqp, 1, di, 0);
    if (e == cudaSuccess) e = cudaMemcpy(ind, di, sizeof(int) * (size_t)nk * nqp, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) rc = ADGA_ECUDA;
  }
  cudaFree(dq); cudaFree(dk); cudaFree(di);
  return rc;
}

extern "C" int adga_generate_q_vol(int nkpx, int nkpy, int nkpz, int nqpx, int nqpy, int nqpz,
                                   int *q_data) {
  if (!q_data || nqpx < 1 || nqpy < 1 || nqpz < 1) return ADGA_EINVAL;
  if (nkpx % nqpx || nkpy % nqpy || nkpz % nqpz) return ADGA_EINVAL;   // config_init check
  int i1 = 0;
  for (int i = 0; i < nqpx; ++i)
    for (int j = 0; j < nqpy; ++j)
      for (int k = 0; k < nqpz; ++k)
        q_data[i1++] = 1 + k * nkpz / nqpz + (j * nkpy / nqpy) * nkpz + (i * nkpx / nqpx) * nkpy * nkpz;
  return 0;
}

extern "C" int adga_create_u(int nd, double U, double V, double J, double *Umat, adga_z *u,
                             adga_z *ut) {
  if (nd < 1 || nd > 16 || !u || !ut) return ADGA_EINVAL;
  std::vector<double> Um((size_t)nd * nd * nd * nd, 0.0);
  auto at = [&](int i, int j, int k, int l) -> double & {
    return Um[i + (size_t)nd * (j + (size_t)nd * (k + (size_t)nd * l))];
  };
  // one atom, all bands correlated, Kanamori (interaction_mode 1)
  for (int i = 0; i < nd; ++i)
    for (int j = 0; j < nd; ++j)
      for (int k = 0; k < nd; ++k)
        for (int l = 0; l < nd; ++l) {
          if (i == j && k == l) {
            if (i == k) { at(i, j, k, l) = U; continue; }
            at(i, j, k, l) = J;
            continue;
          }
          if (i == k && j == l) { at(i, j, k, l) = V; continue; }
          if (i == l && j == k) { at(i, j, k, l) = J; continue; }
        }
  const int nd2 = nd * nd;
  for (int l = 0; l < nd; ++l)
    for (int j = 0; j < nd; ++j) {
      const int i2 = l * nd + j;
      for (int i = 0; i < nd; ++i)
        for (int k = 0; k < nd; ++k) {
          const int i1 = i * nd + k;
          u[i1 + (size_t)i2 * nd2] = {at(i, j, k, l), 0.0};
          ut[i1 + (size_t)i2 * nd2] = {at(i, j, l, k), 0.0};
        }
    }
  if (Umat) memcpy(Umat, Um.data(), sizeof(double) * Um.size());
  return 0;
}
