// Bubble and EOM on the cyclic k mesh through discrete Fourier transforms.
//
// Both k-sums of the loop are cyclic correlations over the k mesh (k - q is
// taken modulo the mesh, src/kq_tools.f90:96-108):
//   chi0^q({i,j},{l,k'}; nu) = -(beta/nkp) sum_k G_il(k, nu) G_k'j(k - q, nu - omega)
//                              (src/one_particle_quant_module.f90:228-290)
//   Sigma_il(k, nu)         += sum_q sum_{j,k'} m_tot({i,j},{l,k'}; nu, q) G_jk'(k - q, nu - omega)
//                              (src/eom_module.f90:210-226)
// With G^(p) = sum_k G(k) e^{-2 pi i p.k / n} (per axis) the first is
//   sum_k A(k) B(k - q) = (1/nkp) sum_p A^(p) B^(-p) e^{+2 pi i p.q / n},
// and the second is (1/nkp) sum_p e^{+2 pi i p.k/n} G^(p) M^(p), M^(p) = sum_q M(q) e^{-2 pi i p.q/n}.
// The q points lie on the sub-mesh q = s.a (s = n/m per axis), so e^{2 pi i p.q/n}
// depends only on p mod m: the bubble folds the products onto the m mesh and
// transforms there, and M^ is an m-mesh transform.  Per omega slice this
// replaces npts.nkp.nd2^2 complex MACs per nu by O(nkp.nd2^2 + m^3 nd2^2 (mx+my+mz));
// the results agree with the direct sums to rounding.
//
// Every transform is a sequence of one-axis passes (k_dft_axis, one output
// element per thread, the axis line read from L1/L2) over arrays laid out
// [batch][x][y][z][component], z fastest like the k index of the .hk file.
#include "ctx.cuh"

__global__ void __launch_bounds__(256)
k_dft_axis(size_t total, int n0, int n1, int n2, int C, int axis, const double2 *__restrict__ tw, double sign,
           const z64 *__restrict__ in, z64 *__restrict__ out) {
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
    size_t r = e / C;
    const int i2 = (int)(r % n2);
    r /= n2;
    const int i1 = (int)(r % n1);
    r /= n1;
    const int i0 = (int)(r % n0);
    int n, idx;
    size_t stride;
    if (axis == 2) { n = n2; idx = i2; stride = C; }
    else if (axis == 1) { n = n1; idx = i1; stride = (size_t)n2 * C; }
    else { n = n0; idx = i0; stride = (size_t)n1 * n2 * C; }
    const z64 *src = in + (e - (size_t)idx * stride);
    double sr = 0.0, si = 0.0;
    int t = 0;
    for (int j = 0; j < n; ++j) {
      const z64 v = src[(size_t)j * stride];
      const double2 w = tw[t];
      const double ws = sign * w.y;
      sr = fma(v.x, w.x, fma(-v.y, ws, sr));
      si = fma(v.x, ws, fma(v.y, w.x, si));
      t += idx;
      if (t >= n) t -= n;
    }
    out[e] = make_double2(sr, si);
  }
}

static unsigned dft_blocks(size_t total) {
  return (unsigned)std::min<size_t>(cdiv_u(total, 256), (size_t)148 * 16);
}

// 3D transform of `batch` arrays (n0, n1, n2, C) from src, ping-ponging between
// x and y (src may be x); returns the buffer that holds the result
z64 *dft3(const z64 *src, z64 *x, z64 *y, int batch, const int n[3], const double2 *const tw[3], int C, double sign,
          cudaStream_t st, cudaError_t *err) {
  const size_t total = (size_t)batch * n[0] * n[1] * n[2] * C;
  const z64 *cur = src;
  *err = cudaSuccess;
  for (int ax = 0; ax < 3 && *err == cudaSuccess; ++ax) {
    if (n[ax] == 1) continue;
    z64 *dst = cur == x ? y : x;
    k_dft_axis<<<dft_blocks(total), 256, 0, st>>>(total, n[0], n[1], n[2], C, ax, tw[ax], sign, cur, dst);
    *err = ADGA_LAUNCH_CHECK();
    cur = dst;
  }
  if (*err == cudaSuccess && cur == src && src != x) {
    *err = cudaMemcpyAsync(x, src, total * sizeof(z64), cudaMemcpyDeviceToDevice, st);
    cur = x;
  }
  return const_cast<z64 *>(cur);
}

// G^(p, nu) of a G table (layout of DevCtx::gtab) into ghat; scratch holds one table
cudaError_t launch_gtable_dft(const DevCtx &c, const z64 *gtab, z64 *ghat, z64 *scratch, cudaStream_t st) {
  const int n[3] = {c.nkpx, c.nkpy, c.nkpz};
  const double2 *tw[3] = {c.dft.twk[0], c.dft.twk[1], c.dft.twk[2]};
  cudaError_t e;
  z64 *res = dft3(gtab, ghat, scratch, c.nnu, n, tw, c.nd2, -1.0, st, &e);
  if (e == cudaSuccess && res != ghat)
    e = cudaMemcpyAsync(ghat, res, sizeof(z64) * c.nnu * c.nkp * c.nd2, cudaMemcpyDeviceToDevice, st);
  return e;
}

// F[inu][p' on the m mesh][a][b] = sum_{p = p' mod m} A^_a(p, nu) B^_b(-p, nu - omega),
// a = i + l nd (G_il), b = k' + j nd (G_k'j); one thread per (inu, p', a)
template <int ND>
__global__ void __launch_bounds__(256)
k_chi0_fold(DevCtx c, int iwb, int nnu_all, const z64 *__restrict__ ghat1, const z64 *__restrict__ ghat2,
            z64 *__restrict__ F) {
  constexpr int ND2 = ND * ND;
  const int mx = c.dft.m[0], my = c.dft.m[1], mz = c.dft.m[2], m3 = mx * my * mz;
  const int sx = c.nkpx / mx, sy = c.nkpy / my, sz = c.nkpz / mz;
  const size_t total = (size_t)nnu_all * m3 * ND2;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
    const int a = (int)(e % ND2);
    const size_t r = e / ND2;
    const int pl = (int)(r % m3), inu = (int)(r / m3);
    const int pz0 = pl % mz, py0 = (pl / mz) % my, px0 = pl / (mz * my);
    const int nu = c.iwstart + inu;
    const z64 *A = ghat1 + (size_t)(nu - c.nu_lo) * c.nkp * ND2;
    const z64 *B = ghat2 + (size_t)(nu - iwb - c.nu_lo) * c.nkp * ND2;
    z64 acc[ND2];
#pragma unroll
    for (int b = 0; b < ND2; ++b) acc[b] = make_double2(0.0, 0.0);
    for (int ax = 0; ax < sx; ++ax) {
      const int px = px0 + ax * mx, nx = px ? c.nkpx - px : 0;
      for (int ay = 0; ay < sy; ++ay) {
        const int py = py0 + ay * my, ny = py ? c.nkpy - py : 0;
        for (int az = 0; az < sz; ++az) {
          const int pz = pz0 + az * mz, nz = pz ? c.nkpz - pz : 0;
          const size_t kp = pz + (size_t)c.nkpz * (py + (size_t)c.nkpy * px);
          const size_t kn = nz + (size_t)c.nkpz * (ny + (size_t)c.nkpy * nx);
          const z64 av = __ldg(A + kp * ND2 + a);
#pragma unroll
          for (int b = 0; b < ND2; ++b) cfma(acc[b], av, __ldg(B + kn * ND2 + b));
        }
      }
    }
    z64 *o = F + e * ND2;
#pragma unroll
    for (int b = 0; b < ND2; ++b) o[b] = acc[b];
  }
}

// chi0_all[p][inu]({i,j},{l,k'}) = fac * F~[inu][q(p)][a = i + l nd][b = k' + j nd]
template <int ND>
__global__ void __launch_bounds__(256)
k_chi0_gather(DevCtx c, const int *__restrict__ qidx, int npts, int nnu_all, double fac, const z64 *__restrict__ F,
              z64 *__restrict__ out) {
  constexpr int ND2 = ND * ND, ND4 = ND2 * ND2;
  const int m3 = c.dft.m[0] * c.dft.m[1] * c.dft.m[2];
  const size_t total = (size_t)npts * nnu_all * ND4;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
    const int o = (int)(e % ND4);
    const size_t r = e / ND4;
    const int inu = (int)(r % nnu_all), p = (int)(r / nnu_all);
    const int o1 = o % ND2, o2 = o / ND2;
    const int i = o1 / ND, j = o1 % ND, l = o2 / ND, kp = o2 % ND;
    const z64 v = F[((size_t)inu * m3 + c.dft.qlin[qidx[p]]) * ND4 + (i + l * ND) * ND2 + (kp + j * ND)];
    out[e] = make_double2(fac * v.x, fac * v.y);
  }
}

// the bubble of a batch of points at one omega by the transform (G^ tables of the
// two factors: ghat1 for G(k, nu), ghat2 for G(k - q, nu - omega))
cudaError_t launch_chi0_dft(const DevCtx &c, int iwb, const int *qidx, int npts, z64 *chi0_all, int nnu_all,
                            const z64 *ghat1, const z64 *ghat2, cudaStream_t st) {
  const int m3 = c.dft.m[0] * c.dft.m[1] * c.dft.m[2];
  const size_t nf = (size_t)nnu_all * m3 * c.nd2;
  const size_t ng = (size_t)npts * nnu_all * c.nd2 * c.nd2;
  const double2 *tw[3] = {c.dft.twm[0], c.dft.twm[1], c.dft.twm[2]};
  const double fac = -c.beta / ((double)c.nkp * (double)c.nkp);
  cudaError_t e = cudaSuccess;
  z64 *res = nullptr;
#define CHI0T(NDD)                                                                                   \
  k_chi0_fold<NDD><<<dft_blocks(nf), 256, 0, st>>>(c, iwb, nnu_all, ghat1, ghat2, c.dft.a);          \
  if ((e = ADGA_LAUNCH_CHECK()) != cudaSuccess) return e;                                             \
  res = dft3(c.dft.a, c.dft.a, c.dft.b, nnu_all, c.dft.m, tw, NDD * NDD * NDD * NDD, 1.0, st, &e);   \
  if (e != cudaSuccess) return e;                                                                     \
  k_chi0_gather<NDD><<<dft_blocks(ng), 256, 0, st>>>(c, qidx, npts, nnu_all, fac, res, chi0_all);
  switch (c.nd) {
    case 1: { CHI0T(1) } break;
    case 2: { CHI0T(2) } break;
    case 3: { CHI0T(3) } break;
    case 4: { CHI0T(4) } break;
    case 5: { CHI0T(5) } break;
    default: return cudaErrorInvalidValue;
  }
#undef CHI0T
  return ADGA_LAUNCH_CHECK();
}

// ---------------------------------------------------------------------------
// EOM
// ---------------------------------------------------------------------------
// Mg[nu][a(q)][c] = m_tot[p][nu][c] for the batch's points (the rest of the m mesh is zero)
__global__ void k_eom_scatter(DevCtx c, const int *__restrict__ qidx, int npts, const z64 *__restrict__ mtot,
                              z64 *__restrict__ Mg) {
  const int nd4 = c.nd2 * c.nd2, m3 = c.dft.m[0] * c.dft.m[1] * c.dft.m[2];
  const size_t total = (size_t)npts * c.iwf * nd4;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
    const int cc = (int)(e % nd4);
    const size_t r = e / nd4;
    const int nu = (int)(r % c.iwf), p = (int)(r / c.iwf);
    Mg[((size_t)nu * m3 + c.dft.qlin[qidx[p]]) * nd4 + cc] = mtot[e];
  }
}

// S[nu][p][i + l nd] = sum_{j,k'} G^_jk'(p, nu - omega) M^[nu][p mod m]({i,j},{l,k'})
template <int ND>
__global__ void __launch_bounds__(256)
k_eom_prod(DevCtx c, int iwb, const z64 *__restrict__ ghat, const z64 *__restrict__ Mh, z64 *__restrict__ S) {
  constexpr int ND2 = ND * ND, ND4 = ND2 * ND2;
  const int mx = c.dft.m[0], my = c.dft.m[1], mz = c.dft.m[2], m3 = mx * my * mz;
  const size_t total = (size_t)c.iwf * c.nkp;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
    const int p = (int)(e % c.nkp), nu = (int)(e / c.nkp);
    const int pz = p % c.nkpz, py = (p / c.nkpz) % c.nkpy, px = p / (c.nkpz * c.nkpy);
    const int pm = pz % mz + mz * (py % my + my * (px % mx));
    const z64 *g = ghat + ((size_t)(nu - iwb - c.nu_lo) * c.nkp + p) * ND2;
    const z64 *M = Mh + ((size_t)nu * m3 + pm) * ND4;
    z64 G[ND2], acc[ND2];
#pragma unroll
    for (int a = 0; a < ND2; ++a) { G[a] = __ldg(g + a); acc[a] = make_double2(0.0, 0.0); }
#pragma unroll
    for (int l = 0; l < ND; ++l)
#pragma unroll
      for (int k2 = 0; k2 < ND; ++k2)
#pragma unroll
        for (int i = 0; i < ND; ++i)
#pragma unroll
          for (int j = 0; j < ND; ++j)
            cfma(acc[i + l * ND], __ldg(M + (i * ND + j) + (l * ND + k2) * ND2), G[j + k2 * ND]);
    z64 *o = S + e * ND2;
#pragma unroll
    for (int a = 0; a < ND2; ++a) o[a] = acc[a];
  }
}

// sigma(k_eom, nu >= 0) += S~[nu][k] / nkp
__global__ void k_eom_add(DevCtx c, const z64 *__restrict__ S, z64 *__restrict__ sigma) {
  const int nd2 = c.nd2, iwf = c.iwf;
  const double f = 1.0 / (double)c.nkp;
  const size_t total = (size_t)c.nkp_eom * iwf * nd2;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
    const int a = (int)(e % nd2);
    const size_t r = e / nd2;
    const int nu = (int)(r % iwf), ik = (int)(r / iwf);
    const int kf = c.keom ? c.keom[ik] - 1 : ik;
    const z64 v = S[((size_t)nu * c.nkp + kf) * nd2 + a];
    z64 &s = sigma[((size_t)ik * 2 * iwf + nu + iwf) * nd2 + a];
    s = make_double2(fma(f, v.x, s.x), fma(f, v.y, s.y));
  }
}

// Sigma(k, nu >= 0) += sum_q m_tot G(k - q, nu - omega) for a batch at one omega by the
// transform (ghat: G^ of the G factor)
cudaError_t launch_eom_dft(const DevCtx &c, int iwb, const int *qidx, int npts, const z64 *mtot, const z64 *ghat,
                           z64 *sigma, cudaStream_t st) {
  const int m3 = c.dft.m[0] * c.dft.m[1] * c.dft.m[2];
  const size_t nd4 = (size_t)c.nd2 * c.nd2;
  const size_t nm = (size_t)c.iwf * m3 * nd4, ns = (size_t)c.iwf * c.nkp;
  const double2 *twm[3] = {c.dft.twm[0], c.dft.twm[1], c.dft.twm[2]};
  const double2 *twk[3] = {c.dft.twk[0], c.dft.twk[1], c.dft.twk[2]};
  const int nk[3] = {c.nkpx, c.nkpy, c.nkpz};
  cudaError_t e = cudaMemsetAsync(c.dft.a, 0, nm * sizeof(z64), st);
  if (e != cudaSuccess) return e;
  const size_t nsc = (size_t)npts * c.iwf * nd4;
  k_eom_scatter<<<dft_blocks(nsc), 256, 0, st>>>(c, qidx, npts, mtot, c.dft.a);
  if ((e = ADGA_LAUNCH_CHECK()) != cudaSuccess) return e;
  z64 *Mh = dft3(c.dft.a, c.dft.a, c.dft.b, c.iwf, c.dft.m, twm, (int)nd4, -1.0, st, &e);
  if (e != cudaSuccess) return e;
  z64 *S = Mh == c.dft.a ? c.dft.b : c.dft.a;
#define EOMT(NDD) k_eom_prod<NDD><<<dft_blocks(ns), 256, 0, st>>>(c, iwb, ghat, Mh, S)
  switch (c.nd) {
    case 1: EOMT(1); break;
    case 2: EOMT(2); break;
    case 3: EOMT(3); break;
    case 4: EOMT(4); break;
    case 5: EOMT(5); break;
    default: return cudaErrorInvalidValue;
  }
#undef EOMT
  if ((e = ADGA_LAUNCH_CHECK()) != cudaSuccess) return e;
  z64 *St = dft3(S, S, Mh, c.iwf, nk, twk, c.nd2, 1.0, st, &e);
  if (e != cudaSuccess) return e;
  const size_t na = (size_t)c.nkp_eom * c.iwf * c.nd2;
  k_eom_add<<<dft_blocks(na), 256, 0, st>>>(c, St, sigma);
  return ADGA_LAUNCH_CHECK();
}
