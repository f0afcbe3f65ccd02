// Common device helpers for the admp_b200 electrostatics kernels (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <math.h>

#include "admp_b200.h"

namespace admp {

constexpr int kOrder = 6;          // PME B-spline order (pme.py:167-169 fixes 6)
constexpr int kStencil = 216;      // 6^3 mesh points per atom
constexpr double kPi = 3.14159265358979323846;
constexpr double kSqrtPi = 1.77245385090551602730;
constexpr int kMaxBatch = 256;     // systems per launch descriptor (by-value kernel parameter, < 32 KB)

template <typename T>
struct Cplx {
  T x, y;
};

// Per-launch error word: kernels never trap; they record the first bad
// condition here and skip the access.  The host reads it after the call.
struct DevError {
  int code;
  int where;
  long long detail;
};

__device__ __forceinline__ void report_error(DevError* e, int code, int where, long long detail) {
  if (e && atomicCAS(&e->code, 0, code) == 0) {
    e->where = where;
    e->detail = detail;
  }
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide sum of `n` doubles per thread into `out` (atomic add); `sh`
// must hold n * 32 doubles.
template <int NV>
__device__ __forceinline__ void block_atomic_sum(double (&v)[NV], double* out, double* sh) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int k = 0; k < NV; ++k) v[k] = warp_sum(v[k]);
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) sh[k * 32 + warp] = v[k];
  }
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      double s = lane < nw ? sh[k * 32 + lane] : 0.0;
      s = warp_sum(s);
      if (lane == 0 && s != 0.0) atomicAdd(out + k, s);
    }
  }
  __syncthreads();
}

// 3x3 inverse and determinant (row-major), double.
__device__ __forceinline__ double inv3(const double* a, double* b) {
  double c00 = a[4] * a[8] - a[5] * a[7];
  double c01 = a[5] * a[6] - a[3] * a[8];
  double c02 = a[3] * a[7] - a[4] * a[6];
  double det = a[0] * c00 + a[1] * c01 + a[2] * c02;
  double id = 1.0 / det;
  b[0] = c00 * id;
  b[1] = (a[2] * a[7] - a[1] * a[8]) * id;
  b[2] = (a[1] * a[5] - a[2] * a[4]) * id;
  b[3] = c01 * id;
  b[4] = (a[0] * a[8] - a[2] * a[6]) * id;
  b[5] = (a[2] * a[3] - a[0] * a[5]) * id;
  b[6] = c02 * id;
  b[7] = (a[1] * a[6] - a[0] * a[7]) * id;
  b[8] = (a[0] * a[4] - a[1] * a[3]) * id;
  return det;
}

template <typename T>
__device__ __forceinline__ void load_box(const T* box, double* b) {
#pragma unroll
  for (int k = 0; k < 9; ++k) b[k] = (double)box[k];
}

// Order-6 cardinal B-spline weights for fractional offset t in [0,1).
// w[k] = M6(t + k), k = 0..5, built by the Cox-de Boor recursion
// M_n(u) = u/(n-1) M_{n-1}(u) + (n-u)/(n-1) M_{n-1}(u-1);  d[k] = M6'(t+k)
// = M5(t+k) - M5(t+k-1).  Mathematically identical to the piecewise
// quintics of recip.py:102-143 evaluated at u0 + s (u0 = t + 3, s = k - 3).
template <typename T>
__device__ __forceinline__ void bspline6(T t, T* w, T* d) {
  T m[6];
  m[0] = t;
  m[1] = T(1) - t;
#pragma unroll
  for (int n = 3; n <= 5; ++n) {
    // from M_{n-1} (entries 0..n-2) to M_n (entries 0..n-1)
    T inv = T(1) / T(n - 1);
    T prev = T(0);
#pragma unroll
    for (int k = 0; k < n; ++k) {
      T cur = k < n - 1 ? m[k] : T(0);
      T u = t + T(k);
      T val = (u * cur + (T(n) - u) * prev) * inv;
      prev = cur;
      m[k] = val;
    }
  }
  // m now holds M5(t+k), k=0..4
  d[0] = m[0];
#pragma unroll
  for (int k = 1; k < 5; ++k) d[k] = m[k] - m[k - 1];
  d[5] = -m[4];
  T prev = T(0);
  const T inv5 = T(1) / T(5);
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    T cur = k < 5 ? m[k] : T(0);
    T u = t + T(k);
    w[k] = (u * cur + (T(6) - u) * prev) * inv5;
    prev = cur;
  }
}

__device__ __forceinline__ int wrap_index(int i, int K) {
  int r = i % K;
  return r < 0 ? r + K : r;
}

// erfc: CUDA's own implementations.
__device__ __forceinline__ double erfc_t(double x) { return erfc(x); }
__device__ __forceinline__ float erfc_t(float x) { return erfcf(x); }
__device__ __forceinline__ double exp_t(double x) { return exp(x); }
__device__ __forceinline__ float exp_t(float x) { return expf(x); }
__device__ __forceinline__ double sqrt_t(double x) { return sqrt(x); }
__device__ __forceinline__ float sqrt_t(float x) { return sqrtf(x); }
__device__ __forceinline__ double rint_t(double x) { return rint(x); }
__device__ __forceinline__ float rint_t(float x) { return rintf(x); }
__device__ __forceinline__ double floor_t(double x) { return floor(x); }
__device__ __forceinline__ float floor_t(float x) { return floorf(x); }
__device__ __forceinline__ double ceil_t(double x) { return ceil(x); }
__device__ __forceinline__ float ceil_t(float x) { return ceilf(x); }

}  // namespace admp

#define ADMP_CUDA_TRY(expr)                                   \
  do {                                                        \
    cudaError_t _e = (expr);                                  \
    if (_e != cudaSuccess) {                                  \
      admp::set_last_cuda_error(_e, #expr, __FILE__, __LINE__); \
      return ADMP_ERR_CUDA;                                   \
    }                                                         \
  } while (0)

namespace admp {
void set_last_cuda_error(cudaError_t e, const char* expr, const char* file, int line);
void set_last_message(const char* fmt, ...);
}  // namespace admp
