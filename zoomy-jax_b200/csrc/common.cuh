// Shared device helpers for the libzb kernels (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <math.h>

#include "zb.h"

namespace zb {

#define ZB_CUDA_TRY(expr)                                  \
  do {                                                     \
    cudaError_t _e = (expr);                               \
    if (_e != cudaSuccess) return ZB_E_CUDA;               \
  } while (0)

static inline int zb_launch_check() {
  return cudaGetLastError() == cudaSuccess ? ZB_OK : ZB_E_CUDA;
}

template <typename T> __device__ __forceinline__ T zmax(T a, T b) { return a > b ? a : b; }
template <typename T> __device__ __forceinline__ T zmin(T a, T b) { return a < b ? a : b; }
// NumPy semantics: np.maximum / np.minimum propagate NaN; fmax would drop it.
__device__ __forceinline__ float nmax(float a, float b) { return (a != a || a > b) ? a : b; }
__device__ __forceinline__ double nmax(double a, double b) { return (a != a || a > b) ? a : b; }
__device__ __forceinline__ float nmin(float a, float b) { return (a != a || a < b) ? a : b; }
__device__ __forceinline__ double nmin(double a, double b) { return (a != a || a < b) ? a : b; }
template <typename T> __device__ __forceinline__ T clip01(T x) {
  return x < T(0) ? T(0) : (x > T(1) ? T(1) : x);
}

// KP-desingularised inverse depth: sqrt(2) h / sqrt(h^4 + max(h, eps)^4)
// (zoomy_jax/fvm/solver_jax.py:291-292).
template <typename T> __device__ __forceinline__ T kp_hinv(T h, T eps) {
  T m = h > eps ? h : eps;
  T h2 = h * h, m2 = m * m;
  return (T(1.4142135623730951) * h) / sqrt(h2 * h2 + m2 * m2);
}

// Non-negative doubles order like their bit patterns: atomicMax on the bits.
// NaN (any sign) compares above +inf, so a non-finite state poisons the max.
__device__ __forceinline__ void atomic_max_pos_double(double* addr, double v) {
  unsigned long long bits = __double_as_longlong(v);
  if (v != v) bits = 0x7FF8000000000000ull | (bits & 0x7FFFFFFFFFFFFFFFull);
  atomicMax(reinterpret_cast<unsigned long long*>(addr), bits);
}

template <typename T> __device__ __forceinline__ bool zfinite(T x) { return isfinite(x); }

// Block-wide max of a double (blockDim.x * blockDim.y threads, <= 1024).
__device__ __forceinline__ double block_max_double(double v, double* sh) {
  const int tid = threadIdx.x + blockDim.x * threadIdx.y;
  const int nthr = blockDim.x * blockDim.y;
  for (int o = 16; o > 0; o >>= 1) v = nmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  if ((tid & 31) == 0) sh[tid >> 5] = v;
  __syncthreads();
  if (tid < 32) {
    double w = (tid < (nthr + 31) / 32) ? sh[tid] : 0.0;
    for (int o = 16; o > 0; o >>= 1) w = nmax(w, __shfl_xor_sync(0xffffffffu, w, o));
    v = w;
  }
  return v;  // valid in thread 0
}

}  // namespace zb
