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
// Hot-path min / max: one FMNMX / DMNMX instruction.  NaN-dropping, unlike
// NumPy's np.maximum; a non-finite state is still detected through the
// owning cell's own update and the NaN-propagating dt reduction (nmax).
__device__ __forceinline__ float fmx(float a, float b) { return fmaxf(a, b); }
__device__ __forceinline__ double fmx(double a, double b) { return fmax(a, b); }
__device__ __forceinline__ float fmn(float a, float b) { return fminf(a, b); }
__device__ __forceinline__ double fmn(double a, double b) { return fmin(a, b); }

__device__ __forceinline__ float clip01(float x) { return __saturatef(x); }
__device__ __forceinline__ double clip01(double x) { return fmin(fmax(x, 0.0), 1.0); }

// float64 quotient, reciprocal square root and square root of the
// shallow-water path: Newton-Raphson refinement of the hardware's approximate
// reciprocal / reciprocal square root (PTX rcp.approx.ftz.f64,
// rsqrt.approx.ftz.f64), each step squaring the seed's relative error, then
// one residual correction in the manner of Markstein (IBM J. Res. Dev. 34(1),
// 1990): q + (a - b q) y for the quotient, s + (x - s s) y / 2 for the root.
// Within one ulp of the exact value for normal positive divisors and
// radicands (zb_newton_check_f64 measures them against IEEE division and
// square root); the callers take a quotient only where its divisor is
// positive.
__device__ __forceinline__ double nrcp(double b) {
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(b));
  double e = fma(-b, y, 1.0);
  y = fma(y, e, y);
  e = fma(-b, y, 1.0);
  return fma(y, e, y);
}
__device__ __forceinline__ double ndiv(double a, double b) {
  const double y = nrcp(b);
  const double q = a * y;
  return fma(fma(-b, q, a), y, q);
}
__device__ __forceinline__ double nrsqrt(double x) {
  double y;
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  const double hx = 0.5 * x;
  double t = fma(-hx * y, y, 0.5);
  y = fma(y, t, y);
  t = fma(-hx * y, y, 0.5);
  return fma(y, t, y);
}
// x >= 0; a negative or NaN x gives NaN, as sqrt does
__device__ __forceinline__ double nsqrt(double x) {
  if (x > 0.0) {
    const double y = nrsqrt(x);
    const double s = x * y;
    return fma(fma(-s, s, x), 0.5 * y, s);
  }
  return x == 0.0 ? x : __longlong_as_double(0x7ff8000000000000LL);
}

// Division of the shallow-water limiter and flux path.  float: __fdividef
// (x * approximate 1/y, at most 2 ulp for |y| < 2^126; the ratios here are
// limiter quotients and the HLL 1/(s_R - s_L)); double: ndiv (one ulp; float64
// parity with the oracle).
__device__ __forceinline__ float adiv(float a, float b) { return __fdividef(a, b); }
__device__ __forceinline__ double adiv(double a, double b) { return ndiv(a, b); }
// Square root of the wave speeds: float sqrtf (approximate under
// -prec-sqrt=false), double nsqrt.
__device__ __forceinline__ float asqrt(float x) { return sqrtf(x); }
__device__ __forceinline__ double asqrt(double x) { return nsqrt(x); }

// Three-operand min / max (NaN-dropping like fmx / fmn; exact, so any grouping
// gives the same bits).  float: the sm_100 three-input PTX forms.
__device__ __forceinline__ float fmx3(float a, float b, float c) {
  float r;
  asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
  return r;
}
__device__ __forceinline__ double fmx3(double a, double b, double c) {
  return fmax(fmax(a, b), c);
}
__device__ __forceinline__ float fmn3(float a, float b, float c) {
  float r;
  asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
  return r;
}
__device__ __forceinline__ double fmn3(double a, double b, double c) {
  return fmin(fmin(a, b), c);
}

// KP-desingularised inverse depth: sqrt(2) h / sqrt(h^4 + max(h, eps)^4)
// (zoomy_jax/fvm/solver_jax.py:291-292).  float: one reciprocal square root;
// double: nrsqrt (float64 parity with the oracle).
__device__ __forceinline__ float kp_hinv(float h, float eps) {
  const float m = fmaxf(h, eps);
  const float h2 = h * h, m2 = m * m;
  return (1.41421356237309515f * h) * rsqrtf(h2 * h2 + m2 * m2);
}
__device__ __forceinline__ double kp_hinv(double h, double eps) {
  const double m = h > eps ? h : eps;
  const double h2 = h * h, m2 = m * m;
  return (1.4142135623730951 * h) * nrsqrt(h2 * h2 + m2 * m2);
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
