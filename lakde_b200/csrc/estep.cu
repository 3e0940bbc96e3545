// Sparse-pair E-step: per-pair log-responsibility numerators (kernel-major
// CSR, one warp per kernel row with the factor in shared memory) and the
// per-point normaliser / threshold / rebalance pass (point-major, one warp per
// point, warp-shuffle reductions, no atomics).
#include "common.cuh"

namespace lakde {

template <typename T, int DP>
struct LogRhoCfg {
  static constexpr int WPB = 4;
  static constexpr int TS = Tri<T>::size(DP);
  // per-warp slice (packed factor + centre) padded to a whole 16-byte vector
  static constexpr int per_warp = ((TS + DP + Tri<T>::V - 1) / Tri<T>::V) * Tri<T>::V;
  static constexpr size_t smem = (size_t)WPB * per_warp * sizeof(T);
};

__device__ __forceinline__ float mul_rn_(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn_(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float add_rn_(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add_rn_(double a, double b) { return __dadd_rn(a, b); }

template <typename T, typename RP, typename CI, int DP>
__global__ void __launch_bounds__(128) estep_logrho_kernel(const RP *__restrict__ rowptr, const CI *__restrict__ col,
                                                           const T *__restrict__ X, int64_t npts, int64_t koff,
                                                           const T *__restrict__ W, const T *__restrict__ nu,
                                                           const T *__restrict__ logdet, T *__restrict__ logrho,
                                                           int64_t N, int D) {
  using C = LogRhoCfg<T, DP>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t n = (int64_t)blockIdx.x * C::WPB + warp;
  if (n >= N) return;
  T *sU = reinterpret_cast<T *>(smem_raw) + warp * C::per_warp;
  T *sxn = sU + C::TS;
  load_tri<T, DP>(sU, W + n * (int64_t)D * D, D, 1, D, true, lane, 32);
  const int64_t self = n + koff;
  for (int d = lane; d < DP; d += 32) sxn[d] = (d < D && self < npts) ? X[self * D + d] : T(0);
  // multivariate digamma, one term per lane
  double md = 0.0;
  for (int i = 1 + lane; i <= D; i += 32) md += digamma_d(0.5 * (double)nu[n] + 0.5 * (1 - i));
  md = warp_sum(md);
  const T cst = (T)(0.5 * (md + D * 0.69314718055994530942 + (double)logdet[n]));
  const T expo = T(-0.5) * nu[n];
  __syncwarp();
  const int64_t start = (int64_t)rowptr[n], end = (int64_t)rowptr[n + 1];
  for (int64_t p = start + lane; p < end; p += 32) {
    const int64_t c = (int64_t)col[p];
    if (c < 0 || c >= npts) {
      logrho[p] = T(NAN);
      continue;
    }
    T delta[DP];
#pragma unroll
    for (int d = 0; d < DP; ++d) delta[d] = (d < D) ? X[c * D + d] - sxn[d] : T(0);
    const T q = quad_tri<T, DP>(sU, delta);
    T lr = add_rn_(mul_rn_(q, expo), cst);
    if (c == self) lr = neg_inf<T>();
    logrho[p] = lr;
  }
}

// Normaliser, threshold and rebalance of one point from its log rho values
// (one warp per point).  Points with at most 128 pairs keep their values in
// registers (four per lane) and read logrho once; longer lists loop.
template <typename T>
struct NormParams {
  int mode;
  T thr, eps, tiny, big;
};

template <typename T>
__device__ __forceinline__ T normaliser_update(T c_old, T rs_old, T lse, int mode) {
  if (mode == 0) return logaddexp(c_old, lse);
  const T old_contrib = log(rs_old) + c_old;
  return logaddexp(logsubexp(c_old, old_contrib), lse);
}

template <typename T>
__device__ __forceinline__ T responsibility(T lr, T c_new, T thr) {
  T rv = exp(lr - c_new);
  if (thr > T(0) && rv <= thr) rv = T(0);
  return rv;
}

template <typename T>
__device__ __forceinline__ T clamp_coeff(T sum, const NormParams<T> &np, T *c_fin, T c_new) {
  sum = sum < np.eps ? np.eps : sum;
  *c_fin = c_new + log(sum);
  T coeff = T(1) / sum;
  return coeff < np.tiny ? np.tiny : (coeff > np.big ? np.big : coeff);
}

template <typename T, typename PI>
__global__ void __launch_bounds__(256) estep_normalise_kernel(const int64_t *__restrict__ cptr,
                                                              const PI *__restrict__ pos,
                                                              const T *__restrict__ logrho, T *__restrict__ r,
                                                              T *__restrict__ c, T *__restrict__ rsum,
                                                              int64_t npts, NormParams<T> np) {
  constexpr int R = 4;
  const int lane = threadIdx.x & 31;
  const int64_t m = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (m >= npts) return;
  const int64_t s = cptr[m], e = cptr[m + 1];
  const T c_old = c[m];
  const T rs_old = rsum[m];
  T c_new, c_fin, coeff, rs = T(0);
  if (e - s <= 32 * R) {
    T v[R];
    int64_t q[R];
#pragma unroll
    for (int k = 0; k < R; ++k) {
      const int64_t p = s + lane + 32 * k;
      q[k] = p < e ? (int64_t)pos[p] : -1;
      v[k] = q[k] >= 0 ? logrho[q[k]] : neg_inf<T>();
    }
    T mx = v[0];
#pragma unroll
    for (int k = 1; k < R; ++k) mx = fmax(mx, v[k]);
    mx = warp_max(mx);
    T se = T(0);
    if (mx != neg_inf<T>()) {
#pragma unroll
      for (int k = 0; k < R; ++k)
        if (q[k] >= 0) se += exp(v[k] - mx);
    }
    se = warp_sum(se);
    const T lse = (mx == neg_inf<T>()) ? mx : mx + log(se);
    c_new = normaliser_update(c_old, rs_old, lse, np.mode);
    T sum = T(0);
#pragma unroll
    for (int k = 0; k < R; ++k) {
      v[k] = q[k] >= 0 ? responsibility(v[k], c_new, np.thr) : T(0);
      sum += v[k];
    }
    sum = warp_sum(sum);
    coeff = clamp_coeff(sum, np, &c_fin, c_new);
#pragma unroll
    for (int k = 0; k < R; ++k) {
      if (q[k] >= 0) {
        const T rv = v[k] * coeff;
        r[q[k]] = rv;
        rs += rv;
      }
    }
  } else {
    T mx = neg_inf<T>();
    for (int64_t p = s + lane; p < e; p += 32) mx = fmax(mx, logrho[pos[p]]);
    mx = warp_max(mx);
    T se = T(0);
    if (mx != neg_inf<T>())
      for (int64_t p = s + lane; p < e; p += 32) se += exp(logrho[pos[p]] - mx);
    se = warp_sum(se);
    const T lse = (mx == neg_inf<T>()) ? mx : mx + log(se);
    c_new = normaliser_update(c_old, rs_old, lse, np.mode);
    T sum = T(0);
    for (int64_t p = s + lane; p < e; p += 32) sum += responsibility(logrho[pos[p]], c_new, np.thr);
    sum = warp_sum(sum);
    coeff = clamp_coeff(sum, np, &c_fin, c_new);
    for (int64_t p = s + lane; p < e; p += 32) {
      const T rv = responsibility(logrho[pos[p]], c_new, np.thr) * coeff;
      r[pos[p]] = rv;
      rs += rv;
    }
  }
  rs = warp_sum(rs);
  if (lane == 0) {
    c[m] = c_fin;
    rsum[m] = rs;
  }
}

// The per-point pass split into stages around cross-shard reductions (kernels
// sharded over devices, every device holding the pairs of its kernels, the
// point-major view cptr / pos over its own pairs).  Between stages the caller
// reduces `red` / `red2` over the shards (max after stage 0, sums after 1, 2
// and 3: rsum).  Per point m, over the local pairs:
//   stage 0: red[m] = max logrho
//   stage 1: red2[m] = sum exp(logrho - red[m])          (red = global max)
//   stage 2: lse = red + log(red2) (global); c_new = normaliser update of
//            (c[m], rsum[m], lse); red[m] = c_new; red2[m] = sum r (thresholded)
//   stage 3: (red = c_new, red2 = global sum) coeff, c[m] = c_fin,
//            r = r * coeff on the local pairs, rsum[m] = local sum of the new r
// The arithmetic is that of estep_normalise_kernel.
template <typename T, typename PI>
__global__ void __launch_bounds__(256) estep_normalise_stage_kernel(const int64_t *__restrict__ cptr,
                                                                    const PI *__restrict__ pos,
                                                                    const T *__restrict__ logrho, T *__restrict__ r,
                                                                    T *__restrict__ c, T *__restrict__ rsum,
                                                                    T *__restrict__ red, T *__restrict__ red2,
                                                                    int64_t npts, int stage, NormParams<T> np) {
  const int lane = threadIdx.x & 31;
  const int64_t m = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (m >= npts) return;
  const int64_t s = cptr[m], e = cptr[m + 1];
  if (stage == 0) {
    T mx = neg_inf<T>();
    for (int64_t p = s + lane; p < e; p += 32) mx = fmax(mx, logrho[pos[p]]);
    mx = warp_max(mx);
    if (lane == 0) red[m] = mx;
  } else if (stage == 1) {
    const T mx = red[m];
    T se = T(0);
    if (mx != neg_inf<T>())
      for (int64_t p = s + lane; p < e; p += 32) se += exp(logrho[pos[p]] - mx);
    se = warp_sum(se);
    if (lane == 0) red2[m] = se;
  } else if (stage == 2) {
    const T mx = red[m];
    const T lse = (mx == neg_inf<T>()) ? mx : mx + log(red2[m]);
    const T c_new = normaliser_update(c[m], rsum[m], lse, np.mode);
    T sum = T(0);
    for (int64_t p = s + lane; p < e; p += 32) sum += responsibility(logrho[pos[p]], c_new, np.thr);
    sum = warp_sum(sum);
    __syncwarp();
    if (lane == 0) {
      red[m] = c_new;
      red2[m] = sum;
    }
  } else {
    const T c_new = red[m];
    T c_fin;
    const T coeff = clamp_coeff(red2[m], np, &c_fin, c_new);
    T rs = T(0);
    for (int64_t p = s + lane; p < e; p += 32) {
      const T rv = responsibility(logrho[pos[p]], c_new, np.thr) * coeff;
      r[pos[p]] = rv;
      rs += rv;
    }
    rs = warp_sum(rs);
    if (lane == 0) {
      c[m] = c_fin;
      rsum[m] = rs;
    }
  }
}

}  // namespace lakde

using namespace lakde;

extern "C" int lakde_estep_normalise_stage(int dtype, int stage, int64_t npts, const void *cptr, const void *pos,
                                           int pos_dtype, const void *logrho, void *r, void *c, void *rsum,
                                           void *red, void *red2, int mode, double threshold, void *stream) {
  clear_error();
  if (npts < 0 || (mode != 0 && mode != 1) || stage < 0 || stage > 3) {
    set_error("estep_normalise_stage: invalid arguments");
    return LAKDE_EINVAL;
  }
  if (npts == 0) return LAKDE_OK;
  if (!cptr || !c || !rsum || !red || !red2) {
    set_error("estep_normalise_stage: null pointer");
    return LAKDE_EINVAL;
  }
  if (int st = bind_device("estep_normalise_stage", {c, cptr, pos, logrho, r, rsum, red, red2})) return st;
  return dispatch_float(dtype, [&](auto t0) {
    using T = decltype(t0);
    return dispatch_index(pos_dtype, [&](auto p0) {
      using PI = decltype(p0);
      const int64_t threads = npts * 32;
      const unsigned blocks = (unsigned)((threads + 255) / 256);
      const T eps = std::is_same<T, float>::value ? (T)1.1920928955078125e-07 : (T)2.220446049250313e-16;
      const T tiny = std::is_same<T, float>::value ? (T)1.1754943508222875e-38 : (T)2.2250738585072014e-308;
      const T big = std::is_same<T, float>::value ? (T)3.4028234663852886e+38 : (T)1.7976931348623157e+308;
      NormParams<T> np{mode, (T)threshold, eps, tiny, big};
      estep_normalise_stage_kernel<T, PI><<<blocks, 256, 0, as_stream(stream)>>>(
          static_cast<const int64_t *>(cptr), static_cast<const PI *>(pos), static_cast<const T *>(logrho),
          static_cast<T *>(r), static_cast<T *>(c), static_cast<T *>(rsum), static_cast<T *>(red),
          static_cast<T *>(red2), npts, stage, np);
      return check_launch("estep_normalise_stage");
    });
  });
}

extern "C" int lakde_estep_logrho(int dtype, int64_t N, int64_t D, int64_t npts, const void *rowptr,
                                  int rowptr_dtype, const void *col, int col_dtype, const void *X,
                                  int64_t kernel_offset, const void *W_triu, const void *nu, const void *logdet_W,
                                  void *logrho, void *stream) {
  clear_error();
  if (N < 0 || D < 1 || npts < 0 || kernel_offset < 0) {
    set_error("estep_logrho: invalid sizes");
    return LAKDE_EINVAL;
  }
  if (N == 0) return LAKDE_OK;
  if (!rowptr || !X || !W_triu || !nu || !logdet_W) {
    set_error("estep_logrho: null pointer");
    return LAKDE_EINVAL;
  }
  if (int st = bind_device("estep_logrho", {logrho, rowptr, col, X, W_triu, nu, logdet_W})) return st;
  return dispatch_float(dtype, [&](auto t0) {
    using T = decltype(t0);
    return dispatch_index(rowptr_dtype, [&](auto r0) {
      using RP = decltype(r0);
      return dispatch_index(col_dtype, [&](auto c0) {
        using CI = decltype(c0);
        return dispatch_dp(D, [&](auto dp) {
          constexpr int DP = decltype(dp)::value;
          using C = LogRhoCfg<T, DP>;
          auto kern = estep_logrho_kernel<T, RP, CI, DP>;
          if (C::smem > 48 * 1024) {
            cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::smem);
            if (e != cudaSuccess) {
              set_error("estep_logrho: %s", cudaGetErrorString(e));
              return (int)LAKDE_ECUDA;
            }
          }
          kern<<<(unsigned)((N + C::WPB - 1) / C::WPB), 32 * C::WPB, C::smem, as_stream(stream)>>>(
              static_cast<const RP *>(rowptr), static_cast<const CI *>(col), static_cast<const T *>(X), npts,
              kernel_offset, static_cast<const T *>(W_triu), static_cast<const T *>(nu),
              static_cast<const T *>(logdet_W), static_cast<T *>(logrho), N, (int)D);
          return check_launch("estep_logrho");
        });
      });
    });
  });
}

extern "C" int lakde_estep_normalise(int dtype, int64_t npts, const void *cptr, const void *pos, int pos_dtype,
                                     const void *logrho, void *r, void *c, void *rsum, int mode, double threshold,
                                     void *stream) {
  clear_error();
  if (npts < 0 || (mode != 0 && mode != 1)) {
    set_error("estep_normalise: invalid arguments");
    return LAKDE_EINVAL;
  }
  if (npts == 0) return LAKDE_OK;
  if (!cptr || !c || !rsum) {
    set_error("estep_normalise: null pointer");
    return LAKDE_EINVAL;
  }
  if (int st = bind_device("estep_normalise", {c, cptr, pos, logrho, r, rsum})) return st;
  return dispatch_float(dtype, [&](auto t0) {
    using T = decltype(t0);
    return dispatch_index(pos_dtype, [&](auto p0) {
      using PI = decltype(p0);
      const int64_t threads = npts * 32;
      const unsigned blocks = (unsigned)((threads + 255) / 256);
      const T eps = std::is_same<T, float>::value ? (T)1.1920928955078125e-07 : (T)2.220446049250313e-16;
      const T tiny = std::is_same<T, float>::value ? (T)1.1754943508222875e-38 : (T)2.2250738585072014e-308;
      const T big = std::is_same<T, float>::value ? (T)3.4028234663852886e+38 : (T)1.7976931348623157e+308;
      NormParams<T> np{mode, (T)threshold, eps, tiny, big};
      estep_normalise_kernel<T, PI><<<blocks, 256, 0, as_stream(stream)>>>(
          static_cast<const int64_t *>(cptr), static_cast<const PI *>(pos), static_cast<const T *>(logrho),
          static_cast<T *>(r), static_cast<T *>(c), static_cast<T *>(rsum), npts, np);
      return check_launch("estep_normalise");
    });
  });
}
