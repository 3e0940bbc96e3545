// Evidence lower bound of LocalKNearestKDE in FP64 (lakde/local_knn_kde.py:256-341
// with the terms of :24-47) in one pass over the kernels and points and a
// deterministic two-level reduction (fixed grid, per-block partials, one
// final block), instead of a few dozen element-wise launches:
//   sum_n [ p_tau_n - q_tau_n + p_lam_n - q_lam_n ]
//   + sum_m ( -D/2 log 2 pi + c_m ) - N log(N - 1)
#include "common.cuh"

namespace lakde {

constexpr int kElboBlocks = 296;
constexpr int kElboThreads = 256;

// sum_{i=1..D} lgamma(a + (1 - i)/2) + D (D - 1)/4 log pi
__device__ __forceinline__ double mvlgamma_d(double a, int D) {
  double s = 0.25 * D * (D - 1) * 1.14472988584940017414;
  for (int i = 1; i <= D; ++i) s += lgamma(a + 0.5 * (1 - i));
  return s;
}

template <typename T>
__global__ void __launch_bounds__(kElboThreads) knn_elbo_kernel(const T *__restrict__ a, const T *__restrict__ b,
                                                                const T *__restrict__ nu,
                                                                const T *__restrict__ logdet_W,
                                                                const T *__restrict__ logdet_s0,
                                                                const T *__restrict__ mm, const T *__restrict__ c,
                                                                int64_t n_kernels, int64_t n_points, int D,
                                                                double a0, double b0, double nu0,
                                                                double *__restrict__ partials) {
  const double LOG2 = 0.69314718055994530942, LOG2PI = 1.83787706640934548356;
  // terms of the prior that do not depend on the kernel (only with kernel
  // terms to add: a points-only call may pass any hyper-parameters)
  double lg_a0 = 0.0, log_b0 = 0.0, log_nu0 = 0.0, mvlg_nu0 = 0.0;
  if (n_kernels > 0) {
    lg_a0 = lgamma(a0);
    log_b0 = log(b0);
    log_nu0 = log(nu0);
    mvlg_nu0 = mvlgamma_d(0.5 * nu0, D);
  }
  double acc = 0.0;
  const int64_t N = n_kernels > n_points ? n_kernels : n_points;
  for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < N; n += (int64_t)gridDim.x * blockDim.x) {
    // index n: the terms of kernel n, then those of point n
    if (n < n_kernels) {
      const double an = (double)a[n], bn = (double)b[n], nun = (double)nu[n];
      const double ldw = (double)logdet_W[n], lds0 = (double)logdet_s0[n], mmn = (double)mm[n];
      const double e_tau = an / bn;
      const double e_log_tau = digamma_d(an) - log(bn);
      const double e_logdet = mvdigamma_d(0.5 * nun, D) + D * LOG2 + ldw;
      const double p_tau = -lg_a0 + a0 * log_b0 + (a0 - 1) * e_log_tau - b0 * e_tau;
      const double q_tau = -lgamma(an) + an * log(bn) + (an - 1) * e_log_tau - bn * e_tau;
      const double B_p = -nu0 / 2 * (D * LOG2 - lds0 - D * e_log_tau - D * log_nu0) - mvlg_nu0;
      const double p_lam = B_p + (nu0 - D - 1) * e_logdet / 2 - e_tau * nu0 * mmn / 2;
      const double B_q = -nun / 2 * (ldw + D * LOG2) - mvlgamma_d(0.5 * nun, D);
      const double q_lam = B_q + (nun - D - 1) * e_logdet / 2 - nun / 2 * D;
      acc += (p_lam - q_lam) + (p_tau - q_tau);
    }
    if (n < n_points) acc += -0.5 * D * LOG2PI + (double)c[n];
  }
  __shared__ double red[kElboThreads / 32];
  acc = warp_sum(acc);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < kElboThreads / 32; ++w) s += red[w];
    partials[blockIdx.x] = s;
  }
}

__global__ void elbo_final_kernel(const double *__restrict__ partials, int n, double tail, double *__restrict__ out) {
  __shared__ double red[32];
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s += partials[i];
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    *out = t + tail;
  }
}

}  // namespace lakde

using namespace lakde;

extern "C" size_t lakde_knn_elbo_workspace(void) { return (size_t)kElboBlocks * sizeof(double); }

extern "C" int lakde_knn_elbo_parts(int dtype, int64_t n_kernels, int64_t n_points, int64_t D, const void *a,
                                    const void *b, const void *nu, const void *logdet_W, const void *logdet_sigma_0,
                                    const void *mm, const void *c, double a_0, double b_0, double nu_0, double tail,
                                    void *workspace, size_t workspace_bytes, double *out, void *stream) {
  clear_error();
  if (n_kernels < 0 || n_points < 0 || D < 1) {
    set_error("knn_elbo_parts: invalid sizes (kernels=%lld, points=%lld, D=%lld)", (long long)n_kernels,
              (long long)n_points, (long long)D);
    return LAKDE_EINVAL;
  }
  if ((n_kernels > 0 && (!a || !b || !nu || !logdet_W || !logdet_sigma_0 || !mm)) || (n_points > 0 && !c) || !out ||
      !workspace) {
    set_error("knn_elbo_parts: null pointer");
    return LAKDE_EINVAL;
  }
  if (workspace_bytes < lakde_knn_elbo_workspace()) {
    set_error("knn_elbo_parts: workspace of %zu bytes needed, %zu given", lakde_knn_elbo_workspace(),
              workspace_bytes);
    return LAKDE_EINVAL;
  }
  if (int st = bind_device("knn_elbo_parts", {out, a, b, nu, logdet_W, logdet_sigma_0, mm, c, workspace})) return st;
  return dispatch_float(dtype, [&](auto t0) {
    using T = decltype(t0);
    double *part = static_cast<double *>(workspace);
    knn_elbo_kernel<T><<<kElboBlocks, kElboThreads, 0, as_stream(stream)>>>(
        static_cast<const T *>(a), static_cast<const T *>(b), static_cast<const T *>(nu),
        static_cast<const T *>(logdet_W), static_cast<const T *>(logdet_sigma_0), static_cast<const T *>(mm),
        static_cast<const T *>(c), n_kernels, n_points, (int)D, a_0, b_0, nu_0, part);
    if (int st = check_launch("knn_elbo")) return st;
    elbo_final_kernel<<<1, 256, 0, as_stream(stream)>>>(part, kElboBlocks, tail, out);
    return check_launch("knn_elbo_final");
  });
}

extern "C" int lakde_knn_elbo(int dtype, int64_t N, int64_t D, const void *a, const void *b, const void *nu,
                              const void *logdet_W, const void *logdet_sigma_0, const void *mm, const void *c,
                              double a_0, double b_0, double nu_0, void *workspace, size_t workspace_bytes,
                              double *out, void *stream) {
  clear_error();
  if (N < 2 || D < 1) {
    set_error("knn_elbo: invalid sizes (N=%lld, D=%lld)", (long long)N, (long long)D);
    return LAKDE_EINVAL;
  }
  if (!a || !b || !nu || !logdet_W || !logdet_sigma_0 || !mm || !c || !out || !workspace) {
    set_error("knn_elbo: null pointer");
    return LAKDE_EINVAL;
  }
  return lakde_knn_elbo_parts(dtype, N, N, D, a, b, nu, logdet_W, logdet_sigma_0, mm, c, a_0, b_0, nu_0,
                              -(double)N * log((double)(N - 1)), workspace, workspace_bytes, out, stream);
}
