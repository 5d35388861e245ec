// Shared device helpers of the ADGA B200 library: complex arithmetic on
// double2 / float2, error plumbing and launch sizes.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstddef>

#define ADGA_HD __host__ __device__ __forceinline__
#define ADGA_D __device__ __forceinline__

typedef double2 z64;
typedef float2 z32;

// ---- complex traits over the two storage types ----
template <typename T> struct cx;
template <> struct cx<z64> {
  typedef double real;
  static ADGA_HD z64 make(double a, double b) { return make_double2(a, b); }
};
template <> struct cx<z32> {
  typedef float real;
  static ADGA_HD z32 make(float a, float b) { return make_float2(a, b); }
};

template <typename T> ADGA_HD T czero() { return cx<T>::make(0, 0); }
template <typename T> ADGA_HD T cadd(T a, T b) { return cx<T>::make(a.x + b.x, a.y + b.y); }
template <typename T> ADGA_HD T csub(T a, T b) { return cx<T>::make(a.x - b.x, a.y - b.y); }
template <typename T> ADGA_HD T cneg(T a) { return cx<T>::make(-a.x, -a.y); }
template <typename T> ADGA_HD T cconj(T a) { return cx<T>::make(a.x, -a.y); }
template <typename T, typename S> ADGA_HD T cscale(T a, S s) { return cx<T>::make(a.x * s, a.y * s); }
template <typename T> ADGA_HD T cmul(T a, T b) {
  return cx<T>::make(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// acc += a * b
template <typename T> ADGA_HD void cfma(T &acc, T a, T b) {
  acc.x = fma(a.x, b.x, acc.x); acc.x = fma(-a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y); acc.y = fma(a.y, b.x, acc.y);
}
// acc -= a * b
template <typename T> ADGA_HD void cfms(T &acc, T a, T b) {
  acc.x = fma(-a.x, b.x, acc.x); acc.x = fma(a.y, b.y, acc.x);
  acc.y = fma(-a.x, b.y, acc.y); acc.y = fma(-a.y, b.x, acc.y);
}
// |re| + |im| (LAPACK's cabs1, used by izamax for pivot selection)
template <typename T> ADGA_HD typename cx<T>::real cabs1(T a) { return fabs(a.x) + fabs(a.y); }

// 1/z with scaling against overflow (Smith's method)
template <typename T> ADGA_HD T crcp(T z) {
  typedef typename cx<T>::real R;
  R a = z.x, b = z.y;
  if (fabs(a) >= fabs(b)) {
    R r = b / a, d = a + b * r;
    return cx<T>::make(R(1) / d, -r / d);
  } else {
    R r = a / b, d = a * r + b;
    return cx<T>::make(r / d, R(-1) / d);
  }
}
// a / b by Smith's method
template <typename T> ADGA_HD T cdiv(T a, T b) {
  typedef typename cx<T>::real R;
  if (fabs(b.x) >= fabs(b.y)) {
    R r = b.y / b.x, d = b.x + b.y * r;
    return cx<T>::make((a.x + a.y * r) / d, (a.y - a.x * r) / d);
  } else {
    R r = b.x / b.y, d = b.x * r + b.y;
    return cx<T>::make((a.x * r + a.y) / d, (a.y * r - a.x) / d);
  }
}

ADGA_HD z32 to32(z64 a) { return make_float2((float)a.x, (float)a.y); }
ADGA_HD z64 to64(z32 a) { return make_double2((double)a.x, (double)a.y); }
template <typename T> ADGA_HD T from64(z64 a);
template <> ADGA_HD z64 from64<z64>(z64 a) { return a; }
template <> ADGA_HD z32 from64<z32>(z64 a) { return to32(a); }
ADGA_HD z64 up64(z64 a) { return a; }
ADGA_HD z64 up64(z32 a) { return to64(a); }

static inline unsigned cdiv_u(size_t a, size_t b) { return (unsigned)((a + b - 1) / b); }

// Raise a kernel's dynamic shared-memory limit on the current device, once per
// (kernel, device): the attribute belongs to the device's context, so a
// process that drives several GPUs sets it on each of them.  Thread-safe.
cudaError_t smem_limit_once(const void *kernel, int bytes);
template <typename K> inline cudaError_t smem_limit(K *kernel, int bytes) {
  return smem_limit_once((const void *)kernel, bytes);
}

// Host-side launch check used after every kernel launch: counts the launch
// (reported in adga_run_stats.kernel_launches) and returns cudaError_t.
#include <atomic>
inline std::atomic<long long> g_adga_launches{0};
#define ADGA_LAUNCH_CHECK() (g_adga_launches.fetch_add(1, std::memory_order_relaxed), cudaGetLastError())
