// Vertex ingest: the compound-index transform of read_vertex
// (src/hdf5_module.f90:629-773).
//
// The local two-particle Green's function of one bosonic frequency arrives
// as w2dynamics stores it, g4(i,j,nu1,k,l,nu2) per channel (Fortran order,
// nu over -W..W-1 of the vertex file's box, before the beta factor the
// reference applies while reading it, :700,711).  The kernel forms
//     chi_loc(i1, i2) = beta g4(i, j, nu1, k, l, nu2)
//     i1 = (nu1 + iwf) nd2 + i nd + j,  i2 = (nu2 + iwf) nd2 + l nd + k
// over the small box nu1, nu2 in -iwf..iwf-1 (:728-742) and adds or removes
// the disconnected terms of the vertex type (:744-770):
//   full G4       dens: -2 beta g_i(nu1) g_l(nu2) for omega = 0, i = j, k = l
//                 inside one correlated subspace; both channels:
//                 -beta g_i(nu1) g_j(nu1 - omega) for nu1 = nu2, i = l, j = k
//                 when the legs are not all in one correlated subspace;
//   connected G4  both channels: -beta g_i(nu1) g_j(nu1 - omega) for
//                 nu1 = nu2, i = l, j = k;
//   chi           as the second full-G4 term.
// One thread per chi_loc element; the result lands in the handle's vertex
// store or in a caller buffer.
#include "ctx.cuh"
#include <algorithm>

__global__ void __launch_bounds__(256)
k_vertex_g4(DevCtx c, int iwb, int vtype, int W, VertexAtoms atoms, const z64 *__restrict__ g4d,
            const z64 *__restrict__ g4m, z64 *__restrict__ chid, z64 *__restrict__ chim) {
  const int N = c.N, nd = c.nd, nd2 = c.nd2, iwf = c.iwf;
  const size_t total = (size_t)N * N;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < total;
       idx += (size_t)gridDim.x * blockDim.x) {
    const int i1 = (int)(idx % N), i2 = (int)(idx / N);
    const int nu1 = i1 / nd2 - iwf, r1 = i1 % nd2, i = r1 / nd, j = r1 % nd;
    const int nu2 = i2 / nd2 - iwf, r2 = i2 % nd2, l = r2 / nd, k = r2 % nd;
    const size_t g = (size_t)i + nd * ((size_t)j + nd * ((size_t)(nu1 + W) +
                     2 * (size_t)W * ((size_t)k + nd * ((size_t)l + nd * (size_t)(nu2 + W)))));
    z64 vd = __ldg(g4d + g), vm = __ldg(g4m + g);
    vd.x *= c.beta; vd.y *= c.beta;
    vm.x *= c.beta; vm.y *= c.beta;
    const int ai = atoms.a[i];
    const bool cor = ai != 0 && ai == atoms.a[j] && atoms.a[k] == atoms.a[l] && ai == atoms.a[l];
    auto gl = [&](int nu, int band) { return c.giw[(nu + c.iwmax) + band * 2 * c.iwmax]; };
    const bool bubble = nu1 == nu2 && i == l && j == k;
    if (vtype == ADGA_VERTEX_FULL_G4) {
      if (iwb == 0 && i == j && k == l && cor) {
        const z64 t = cmul(make_double2(2.0 * c.beta * gl(nu1, i).x, 2.0 * c.beta * gl(nu1, i).y), gl(nu2, l));
        vd = csub(vd, t);
      }
      if (bubble && !cor) {
        const z64 t = cmul(make_double2(c.beta * gl(nu1, i).x, c.beta * gl(nu1, i).y), gl(nu2 - iwb, j));
        vd = csub(vd, t);
        vm = csub(vm, t);
      }
    } else if (vtype == ADGA_VERTEX_CONNECTED_G4 || (vtype == ADGA_VERTEX_CHI_G4 && !cor)) {
      if (bubble) {
        const z64 t = cmul(make_double2(c.beta * gl(nu1, i).x, c.beta * gl(nu1, i).y), gl(nu2 - iwb, j));
        vd = csub(vd, t);
        vm = csub(vm, t);
      }
    }
    chid[idx] = vd;
    chim[idx] = vm;
  }
}

cudaError_t launch_vertex_g4(const DevCtx &c, int iwb, int vtype, int W, const VertexAtoms &atoms,
                             const z64 *g4d, const z64 *g4m, z64 *chid, z64 *chim, cudaStream_t st) {
  const size_t total = (size_t)c.N * c.N;
  const int blocks = (int)std::min<size_t>(cdiv_u(total, 256), 148 * 16);
  k_vertex_g4<<<blocks, 256, 0, st>>>(c, iwb, vtype, W, atoms, g4d, g4m, chid, chim);
  return ADGA_LAUNCH_CHECK();
}

// ---------------------------------------------------------------------------
// External three-leg vertex: the transform of read_threeleg
// (src/hdf5_module.f90:860-880).  g3(a,b,c,d, m) (Fortran order, m over
// 0..2*n3iwf-1 = Matsubara -n3iwf..n3iwf-1, before the beta factor of
// :829,838) -> gamma^w(i1, i2), i1 = i nd + j, i2 = (nu + iwf) nd2 + k nd + l:
//     gamma = beta g3(k, l, j, i, nu)
//           + 2 beta (1 - n_i) G_k(nu)          (dens, omega = 0, i = j, k = l)
//           + G_k(nu) G_l(nu - omega)           (i = k, j = l)
// each term in one correlated subspace only, then divided there by
// -G_k(nu) G_l(nu - omega).  One thread per gamma element.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
k_threeleg(DevCtx c, int iwb, int n3iwf, VertexAtoms atoms, const z64 *__restrict__ g3d,
           const z64 *__restrict__ g3m, z64 *__restrict__ gd, z64 *__restrict__ gm) {
  const int nd = c.nd, nd2 = c.nd2, N = c.N;
  const size_t total = (size_t)nd2 * N;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < total;
       idx += (size_t)gridDim.x * blockDim.x) {
    const int i1 = (int)(idx % nd2), i2 = (int)(idx / nd2);
    const int i = i1 / nd, j = i1 % nd;
    const int w = i2 / nd2, r = i2 % nd2, k = r / nd, l = r % nd;
    const int nu = w - c.iwf;
    const size_t g = (size_t)k + nd * ((size_t)l + nd * ((size_t)j + nd * ((size_t)i + nd * (size_t)(n3iwf + nu))));
    z64 vd = __ldg(g3d + g), vm = __ldg(g3m + g);
    vd.x *= c.beta; vd.y *= c.beta;
    vm.x *= c.beta; vm.y *= c.beta;
    const int ai = atoms.a[i];
    const bool cor = ai != 0 && ai == atoms.a[j] && atoms.a[k] == atoms.a[l] && ai == atoms.a[l];
    if (cor) {
      const z64 gk = c.giw[(nu + c.iwmax) + k * 2 * c.iwmax];
      const z64 gl = c.giw[(nu - iwb + c.iwmax) + l * 2 * c.iwmax];
      if (i == j && k == l && iwb == 0) {
        const z64 one_n = make_double2(1.0 - c.ndmft[i].x, -c.ndmft[i].y);
        const z64 t = cmul(make_double2(2.0 * c.beta * one_n.x, 2.0 * c.beta * one_n.y), gk);
        vd = cadd(vd, t);
      }
      const z64 gg = cmul(gk, gl);
      if (i == k && j == l) {
        vd = cadd(vd, gg);
        vm = cadd(vm, gg);
      }
      const z64 den = make_double2(-gg.x, -gg.y);
      vd = cdiv(vd, den);
      vm = cdiv(vm, den);
    }
    gd[idx] = vd;
    gm[idx] = vm;
  }
}

cudaError_t launch_threeleg(const DevCtx &c, int iwb, int n3iwf, const VertexAtoms &atoms, const z64 *g3d,
                            const z64 *g3m, z64 *gd, z64 *gm, cudaStream_t st) {
  const size_t total = (size_t)c.nd2 * c.N;
  k_threeleg<<<(int)std::min<size_t>(cdiv_u(total, 256), 148 * 16), 256, 0, st>>>(c, iwb, n3iwf, atoms, g3d,
                                                                                  g3m, gd, gm);
  return ADGA_LAUNCH_CHECK();
}

// 1 + gamma^w from a given gamma^w (src/main.F90:617-625)
__global__ void k_one_plus_gamma(int N, int nd2, const z64 *gam, z64 *opg) {
  const size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (idx >= (size_t)nd2 * N) return;
  const int i1 = (int)(idx % nd2), cc = (int)(idx / nd2);
  z64 s = gam[idx];
  if (cc % nd2 == i1) s.x += 1.0;
  opg[idx] = s;
}

cudaError_t launch_one_plus_gamma(const DevCtx &c, const z64 *gam, z64 *opg, cudaStream_t st) {
  const size_t total = (size_t)c.nd2 * c.N;
  k_one_plus_gamma<<<cdiv_u(total, 256), 256, 0, st>>>(c.N, c.nd2, gam, opg);
  return ADGA_LAUNCH_CHECK();
}

// ---------------------------------------------------------------------------
// External local susceptibility: the transform of read_chi_loc
// (src/hdf5_module.f90:958-993).  chi(a,b,c,d, m) (m over 0..2*n2iwb =
// bosonic -n2iwb..n2iwb) -> chi_loc(i1, i2, omega), i1 = i nd + j,
// i2 = k nd + l: chi(i, j, l, k, omega), minus 2 beta (1 - n_i)(1 - n_k) at
// omega = 0 in the dens channel (i = j, k = l, one correlated subspace) and,
// when `extend` (more than one impurity or uncorrelated bands), minus the
// lattice bubble sum_nu G_i(nu) G_j(nu - omega) / beta of the legs outside a
// common correlated subspace (i = k, j = l).  One thread per element.
// ---------------------------------------------------------------------------
__global__ void k_chi_loc_ext(DevCtx c, int n2iwb, VertexAtoms atoms, int extend, const z64 *__restrict__ rd,
                              const z64 *__restrict__ rm, z64 *__restrict__ od, z64 *__restrict__ om) {
  const int nd = c.nd, nd2 = c.nd2, nw = 2 * c.iwb + 1;
  const size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (idx >= (size_t)nd2 * nd2 * nw) return;
  const int i1 = (int)(idx % nd2), i2 = (int)((idx / nd2) % nd2), wi = (int)(idx / ((size_t)nd2 * nd2));
  const int i = i1 / nd, j = i1 % nd, k = i2 / nd, l = i2 % nd, w = wi - c.iwb;
  const size_t g = (size_t)i + nd * ((size_t)j + nd * ((size_t)l + nd * ((size_t)k + nd * (size_t)(n2iwb + w))));
  z64 vd = rd[g], vm = rm[g];
  const int ai = atoms.a[i];
  const bool cor = ai != 0 && ai == atoms.a[j] && atoms.a[k] == atoms.a[l] && ai == atoms.a[l];
  if (cor && i == j && k == l && w == 0) {
    const z64 a = make_double2(1.0 - c.ndmft[i].x, -c.ndmft[i].y), b = make_double2(1.0 - c.ndmft[k].x, -c.ndmft[k].y);
    const z64 t = cmul(make_double2(2.0 * c.beta * a.x, 2.0 * c.beta * a.y), b);
    vd = csub(vd, t);
  }
  if (extend && !cor && i == k && j == l) {
    for (int n = -c.iwmax + c.iwb; n < c.iwmax - c.iwb; ++n) {
      const z64 t = cmul(c.giw[(n + c.iwmax) + i * 2 * c.iwmax], c.giw[(n - w + c.iwmax) + j * 2 * c.iwmax]);
      vd = csub(vd, make_double2(t.x / c.beta, t.y / c.beta));
      vm = csub(vm, make_double2(t.x / c.beta, t.y / c.beta));
    }
  }
  od[idx] = vd;
  om[idx] = vm;
}

cudaError_t launch_chi_loc_ext(const DevCtx &c, int n2iwb, const VertexAtoms &atoms, int extend, const z64 *rd,
                               const z64 *rm, z64 *od, z64 *om, cudaStream_t st) {
  const size_t total = (size_t)c.nd2 * c.nd2 * (2 * c.iwb + 1);
  k_chi_loc_ext<<<cdiv_u(total, 128), 128, 0, st>>>(c, n2iwb, atoms, extend, rd, rm, od, om);
  return ADGA_LAUNCH_CHECK();
}
