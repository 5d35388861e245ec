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
