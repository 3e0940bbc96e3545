// Shared helpers of the lakde_b200 kernels: status handling, dtype dispatch,
// padded dimensions, packed triangular layouts and small math routines.
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <initializer_list>
#include <type_traits>

#include "../../include/lakde_b200.h"

namespace lakde {

// Records a printf-style message as this thread's last error.
void set_error(const char *fmt, ...);
void clear_error();

// Checks the launch just issued (configuration errors only; asynchronous
// execution errors surface on the caller's next synchronisation).
int check_launch(const char *what);

// Makes the device holding the given buffers current for this library (the
// reference ops call cudaSetDevice(input.get_device())), and rejects host or
// unregistered pointers and buffers spread over several devices.  Null
// pointers are skipped.
int bind_device(const char *what, std::initializer_list<const void *> ptrs);

inline cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }

// Current value of a launch-choice knob for dimension D (lakde_tuning_set).
int tuning(int knob, int64_t D);

// Largest D handled by the register / shared-memory kernels.
constexpr int kMaxDim = 64;

// Padded dimensions the kernels are instantiated for.
template <typename F>
int dispatch_dp(int64_t D, F &&f) {
  if (D <= 2) return f(std::integral_constant<int, 2>{});
  if (D <= 4) return f(std::integral_constant<int, 4>{});
  if (D <= 8) return f(std::integral_constant<int, 8>{});
  if (D <= 16) return f(std::integral_constant<int, 16>{});
  if (D <= 24) return f(std::integral_constant<int, 24>{});
  if (D <= 32) return f(std::integral_constant<int, 32>{});
  if (D <= 48) return f(std::integral_constant<int, 48>{});
  if (D <= 64) return f(std::integral_constant<int, 64>{});
  set_error("D=%lld exceeds the supported maximum of %d", (long long)D, kMaxDim);
  return LAKDE_EUNSUPPORTED;
}

template <typename F>
int dispatch_float(int dtype, F &&f) {
  if (dtype == LAKDE_F32) return f(float{});
  if (dtype == LAKDE_F64) return f(double{});
  set_error("unsupported value dtype code %d (expected F32 or F64)", dtype);
  return LAKDE_EDTYPE;
}

template <typename F>
int dispatch_index(int dtype, F &&f) {
  if (dtype == LAKDE_I32) return f(int32_t{});
  if (dtype == LAKDE_I64) return f(int64_t{});
  set_error("unsupported index dtype code %d (expected I32 or I64)", dtype);
  return LAKDE_EDTYPE;
}

// ---------------------------------------------------------------------------
// Packed upper-triangular layout, column by column: column i holds rows
// 0..i, padded to a multiple of one 16-byte vector so every column starts
// aligned and can be read with vector loads.
// ---------------------------------------------------------------------------
template <typename T>
struct Tri {
  static constexpr int V = 16 / sizeof(T);
  __host__ __device__ static constexpr int col_len(int i) { return ((i + 1 + V - 1) / V) * V; }
  // sum_{c<i} col_len(c) = V * (V q (q+1)/2 + r (q+1)) with i = qV + r
  __host__ __device__ static constexpr int col_off(int i) {
    return V * (V * (i / V) * (i / V + 1) / 2 + (i % V) * (i / V + 1));
  }
  __host__ __device__ static constexpr int size(int DP) { return col_off(DP); }
};

template <typename T> struct Vec;
template <> struct Vec<float> { using type = float4; };
template <> struct Vec<double> { using type = double2; };

// q = || U^T delta ||^2 for an upper-triangular U held in the packed layout.
template <typename T, int DP>
__device__ __forceinline__ T quad_tri(const T *__restrict__ sU, const T (&delta)[DP]) {
  constexpr int V = Tri<T>::V;
  using VT = typename Vec<T>::type;
  T q = T(0);
  int off = 0;
#pragma unroll
  for (int i = 0; i < DP; ++i) {
    T y = T(0);
#pragma unroll
    for (int j = 0; j <= i; j += V) {
      VT u = *reinterpret_cast<const VT *>(sU + off + j);
      const T *uu = reinterpret_cast<const T *>(&u);
#pragma unroll
      for (int v = 0; v < V; ++v) {
        if (j + v <= i) y = fma(uu[v], delta[j + v], y);
      }
    }
    q = fma(y, y, q);
    off += Tri<T>::col_len(i);
  }
  return q;
}

// Same quad form, also returning z = U^T delta (for gradients).
template <typename T, int DP>
__device__ __forceinline__ T quad_tri_z(const T *__restrict__ sU, const T (&delta)[DP], T (&z)[DP]) {
  constexpr int V = Tri<T>::V;
  using VT = typename Vec<T>::type;
  T q = T(0);
  int off = 0;
#pragma unroll
  for (int i = 0; i < DP; ++i) {
    T y = T(0);
#pragma unroll
    for (int j = 0; j <= i; j += V) {
      VT u = *reinterpret_cast<const VT *>(sU + off + j);
      const T *uu = reinterpret_cast<const T *>(&u);
#pragma unroll
      for (int v = 0; v < V; ++v) {
        if (j + v <= i) y = fma(uu[v], delta[j + v], y);
      }
    }
    z[i] = y;
    q = fma(y, y, q);
    off += Tri<T>::col_len(i);
  }
  return q;
}

// Cooperative copy of W_triu[n] (upper triangle of a [D,D] block with the
// given row / column strides) into the packed layout, zero padded to DP.
// Consecutive threads read consecutive columns of one row.
template <typename T, int DP>
__device__ __forceinline__ void load_tri(T *__restrict__ sU, const T *__restrict__ W, int64_t s_row,
                                         int64_t s_col, int D, bool valid, int tid, int nthreads) {
  for (int e = tid; e < DP * DP; e += nthreads) {
    const int j = e / DP, i = e % DP;  // row j, column i
    if (j >= Tri<T>::col_len(i)) continue;
    T v = T(0);
    if (valid && j <= i && i < D) v = W[j * s_row + i * s_col];
    sU[Tri<T>::col_off(i) + j] = v;
  }
}

// ---------------------------------------------------------------------------
// math
// ---------------------------------------------------------------------------

// Digamma psi(x) for x > 0 in double precision: upward recurrence to x >= 6,
// then the Stirling asymptotic series
//   psi(x) ~ ln x - 1/(2x) - sum_k B_2k / (2k x^2k),  B_2k = 1/6, -1/30, 1/42, -1/30, 5/66.
// Round to the nearest tf32, ties away from zero (10 explicit mantissa bits;
// the low 13 bits zero): add half of the dropped range to the magnitude bits
// and clear them.  Two integer ALU operations; finite inputs far below
// FLT_MAX (centred differences and inverse factors) cannot carry into the
// exponent's all-ones pattern.
__device__ __forceinline__ float tf32_rna(float x) {
  return __uint_as_float((__float_as_uint(x) + 0x1000u) & 0xFFFFE000u);
}

__device__ __forceinline__ double digamma_d(double x) {
  if (!(x > 0.0)) return nan("");
  double acc = 0.0;
  while (x < 6.0) {
    acc -= 1.0 / x;
    x += 1.0;
  }
  const double f = 1.0 / (x * x);
  const double series =
      f * (1.0 / 12 - f * (1.0 / 120 - f * (1.0 / 252 - f * (1.0 / 240 - f * (1.0 / 132)))));
  return acc + log(x) - 0.5 / x - series;
}

// sum_{i=1..D} psi(a + (1 - i)/2)
__device__ __forceinline__ double mvdigamma_d(double a, int D) {
  double s = 0.0;
  for (int i = 1; i <= D; ++i) s += digamma_d(a + 0.5 * (1 - i));
  return s;
}

template <typename T> __device__ __forceinline__ T neg_inf() { return -INFINITY; }

template <typename T>
__device__ __forceinline__ T warp_max(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// log(exp(a) + exp(b)) with -inf handling
template <typename T>
__device__ __forceinline__ T logaddexp(T a, T b) {
  T m = fmax(a, b);
  if (m == neg_inf<T>()) return m;
  return m + log1p(exp(-fabs(a - b)));
}

// a + log1p(max(-exp(b - a), -1))  (lakde/linalg_util.py:41-42)
template <typename T>
__device__ __forceinline__ T logsubexp(T a, T b) {
  T e = -exp(b - a);
  e = (e < T(-1)) ? T(-1) : e;  // NaN propagates like torch.clamp_min
  return a + log1p(e);
}

}  // namespace lakde
