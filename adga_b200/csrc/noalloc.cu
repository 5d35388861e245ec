// adga_inverse_matrix_z_noalloc: the GPU matrix inverse for callers that
// must not allocate device memory.
//
// Some callers cannot call cudaMalloc: a host program whose device memory is
// owned by another allocator (a pool or framework that hands out pointers but
// forbids the library from growing the footprint), code running where an
// allocation would synchronise the device or break a memory budget.  This
// entry point takes the matrix and the result in device memory the caller
// already owns and keeps every intermediate -- the augmented matrix [M | I],
// the pivots, the LAPACK-style info and the inverted diagonal blocks of the
// blocked LU -- in one file-scope __device__ array of fixed size.  Every GPU
// that loads the library holds that array (NOALLOC_SCRATCH_BYTES, about
// 2.6 MB) until the process exits.
//
// Limits and rules:
//   * n <= ADGA_NOALLOC_MAX_N (256); larger n is rejected with ADGA_EINVAL.
//   * The first call on a device looks up the array's device address with
//     cudaGetSymbolAddress (once per device, that device current); make that
//     first call before any stream capture on the device.
//   * All calls share the one array, which keeps the last call's contents:
//     each call rewrites the whole augmented matrix and clears info.  Calls
//     that overlap on the GPU (different streams, or threads) race on it.
//   * Nothing here calls cudaMalloc, cudaFree or an allocating library routine.
#include "adga.h"
#include "lu.cuh"
#include <mutex>

namespace {

constexpr int NA_MAX_N = ADGA_NOALLOC_MAX_N;
constexpr int NA_NB = 64;
constexpr int NA_STEPS = (NA_MAX_N + NA_NB - 1) / NA_NB;
constexpr size_t NA_T_BYTES = sizeof(z64) * (size_t)NA_MAX_N * 2 * NA_MAX_N;   // [M | I]
constexpr size_t NA_BLK_BYTES = sizeof(z64) * (size_t)NA_STEPS * NA_NB * NA_NB;  // Linv or Uinv
constexpr size_t NA_PIV_BYTES = 256 * ((sizeof(int) * NA_MAX_N + 255) / 256);
constexpr size_t NA_OFF_LINV = NA_T_BYTES;
constexpr size_t NA_OFF_UINV = NA_OFF_LINV + NA_BLK_BYTES;
constexpr size_t NA_OFF_PIV = NA_OFF_UINV + NA_BLK_BYTES;
constexpr size_t NA_OFF_INFO = NA_OFF_PIV + NA_PIV_BYTES;
constexpr size_t NA_OFF_RMAP = NA_OFF_INFO + 256;
constexpr size_t NOALLOC_SCRATCH_BYTES = NA_OFF_RMAP + 256 * ((sizeof(int) * RMAP_STRIDE + 255) / 256);
static_assert(NA_OFF_LINV % 256 == 0 && NA_OFF_PIV % 256 == 0 && NA_OFF_INFO % 256 == 0,
              "scratch regions must stay 256-byte aligned");

// the scratch: one per device, lives until the process exits
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

constexpr int MAX_DEVICES = 64;
std::mutex g_mu;
void *g_dev_ptr[MAX_DEVICES] = {nullptr};

// T[:, 0:n] = M, T[:, n:2n] = I  (column-major, ld = n)
__global__ void k_noalloc_fill(const z64 *__restrict__ Min, z64 *__restrict__ T, int n) {
  const size_t total = (size_t)n * 2 * n;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total;
       e += (size_t)gridDim.x * blockDim.x) {
    const size_t col = e / n, row = e % n;
    z64 v;
    if (col < (size_t)n) v = Min[e];
    else v = make_double2((col - n) == row ? 1.0 : 0.0, 0.0);
    T[e] = v;
  }
}

}  // namespace

extern "C" int adga_inverse_matrix_z_noalloc(const adga_z *M_dev, adga_z *Minv_dev, int n,
                                             int *ierr, void *stream) {
  if (!M_dev || !Minv_dev || n < 1) return ADGA_EINVAL;
  if (n > NA_MAX_N) return ADGA_EINVAL;     // beyond the static scratch
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAX_DEVICES) return ADGA_ECUDA;
  void *base;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_dev_ptr[dev]) {
      void *p = nullptr;
      if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return ADGA_ECUDA;
      g_dev_ptr[dev] = p;
    }
    base = g_dev_ptr[dev];
  }
  cudaStream_t st = (cudaStream_t)stream;
  unsigned char *sb = (unsigned char *)base;
  z64 *T = (z64 *)sb;
  int *ipiv = (int *)(sb + NA_OFF_PIV);
  int *info = (int *)(sb + NA_OFF_INFO);
  const size_t strideM = (size_t)n * 2 * n;
  LUBatch lb{n, 2 * n, 1, NA_NB, strideM, ipiv, info, sb + NA_OFF_LINV, sb + NA_OFF_UINV,
             (int *)(sb + NA_OFF_RMAP)};
  cudaError_t e = cudaMemsetAsync(info, 0, sizeof(int), st);
  if (e == cudaSuccess) {
    k_noalloc_fill<<<cdiv_u(strideM, 256) < 1024 ? cdiv_u(strideM, 256) : 1024, 256, 0, st>>>(
        (const z64 *)M_dev, T, n);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = lu_factor<z64>(T, lb, false, nullptr, nullptr, st);
  if (e == cudaSuccess) e = lu_backsolve<z64>(T, lb, T + (size_t)n * n, strideM, n, n, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(Minv_dev, T + (size_t)n * n, sizeof(z64) * n * n, cudaMemcpyDeviceToDevice, st);
  // the info is always read back (the call waits for the stream), so the
  // return value reports a singular matrix whether or not ierr is given
  int hinfo = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&hinfo, info, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return ADGA_ECUDA;
  if (ierr) *ierr = hinfo;
  return hinfo > 0 ? hinfo : 0;
}
