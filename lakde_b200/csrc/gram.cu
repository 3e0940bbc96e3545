// Weighted Gram sum of the hierarchical model's shared-precision update in
// FP64 (lakde/local_hierarchical_kde.py:293-297):
//   out = sum_n w_n W_triu_n W_triu_n^T        (D x D, symmetric)
// straight from the float32 (or float64) factors, without a float64 copy of
// all of them: each CTA walks a contiguous chunk of kernels, stages W_triu_n
// in shared memory and accumulates its share of the lower triangle in FP64
// registers; the per-CTA partials are summed in a fixed order by one block,
// so the result does not depend on scheduling.
#include "common.cuh"

namespace lakde {

constexpr int kGramBlocks = 296;
constexpr int kGramThreads = 256;
constexpr int kGramPerThread = (64 * 65 / 2 + kGramThreads - 1) / kGramThreads;  // 9 lower entries

template <typename T>
__global__ void __launch_bounds__(kGramThreads) gram_partial_kernel(const T *__restrict__ W, const T *__restrict__ w,
                                                                   int64_t N, int D, int64_t chunk,
                                                                   double *__restrict__ partials) {
  __shared__ double sW[64 * 65];  // row i at i * (D + 1): padded against bank conflicts
  const int tri = D * (D + 1) / 2;
  const int ld = D + 1;
  int ei[kGramPerThread], ek[kGramPerThread];
  double acc[kGramPerThread];
#pragma unroll
  for (int s = 0; s < kGramPerThread; ++s) {
    const int e = threadIdx.x + s * kGramThreads;
    int i = 0;
    while ((i + 1) * (i + 2) / 2 <= e) ++i;
    ei[s] = e < tri ? i : -1;
    ek[s] = e < tri ? e - i * (i + 1) / 2 : 0;
    acc[s] = 0.0;
  }
  const int64_t n0 = (int64_t)blockIdx.x * chunk;
  const int64_t n1 = (n0 + chunk < N) ? n0 + chunk : N;
  for (int64_t n = n0; n < n1; ++n) {
    const T *Wn = W + n * (int64_t)D * D;
    __syncthreads();
    for (int e = threadIdx.x; e < D * D; e += kGramThreads) sW[(e / D) * ld + e % D] = (double)Wn[e];
    __syncthreads();
    const double wn = (double)w[n];
#pragma unroll
    for (int s = 0; s < kGramPerThread; ++s) {
      if (ei[s] < 0) continue;
      // (W W^T)_ik = sum_j W_ij W_kj, W upper: j >= max(i, k) = i (k <= i)
      const double *ri = sW + ei[s] * ld, *rk = sW + ek[s] * ld;
      double d = 0.0;
      for (int j = ei[s]; j < D; ++j) d = fma(ri[j], rk[j], d);
      acc[s] = fma(wn, d, acc[s]);
    }
  }
#pragma unroll
  for (int s = 0; s < kGramPerThread; ++s) {
    const int e = threadIdx.x + s * kGramThreads;
    if (e < tri) partials[(int64_t)blockIdx.x * tri + e] = acc[s];
  }
}

__global__ void gram_final_kernel(const double *__restrict__ partials, int nparts, int D, double *__restrict__ out) {
  const int tri = D * (D + 1) / 2;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < tri; e += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int p = 0; p < nparts; ++p) s += partials[(int64_t)p * tri + e];
    int i = 0;
    while ((i + 1) * (i + 2) / 2 <= e) ++i;
    const int k = e - i * (i + 1) / 2;
    out[i * D + k] = s;
    out[k * D + i] = s;
  }
}

}  // namespace lakde

using namespace lakde;

extern "C" size_t lakde_weighted_gram_workspace(int64_t D) {
  if (D < 1 || D > kMaxDim) return 0;
  return (size_t)kGramBlocks * (size_t)(D * (D + 1) / 2) * sizeof(double);
}

extern "C" int lakde_weighted_gram(int dtype, int64_t N, int64_t D, const void *W_triu, const void *w, double *out,
                                   void *workspace, size_t workspace_bytes, void *stream) {
  clear_error();
  if (N < 0 || D < 1 || D > kMaxDim) {
    set_error("weighted_gram: invalid sizes (N=%lld, D=%lld)", (long long)N, (long long)D);
    return D > kMaxDim ? LAKDE_EUNSUPPORTED : LAKDE_EINVAL;
  }
  if (!out || !workspace || (N > 0 && (!W_triu || !w))) {
    set_error("weighted_gram: null pointer");
    return LAKDE_EINVAL;
  }
  if (workspace_bytes < lakde_weighted_gram_workspace(D)) {
    set_error("weighted_gram: workspace of %zu bytes needed, %zu given", lakde_weighted_gram_workspace(D),
              workspace_bytes);
    return LAKDE_EINVAL;
  }
  if (int st = bind_device("weighted_gram", {out, W_triu, w, workspace})) return st;
  return dispatch_float(dtype, [&](auto t0) {
    using T = decltype(t0);
    const int64_t chunk = N > 0 ? (N + kGramBlocks - 1) / kGramBlocks : 1;
    double *part = static_cast<double *>(workspace);
    gram_partial_kernel<T><<<kGramBlocks, kGramThreads, 0, as_stream(stream)>>>(
        static_cast<const T *>(W_triu), static_cast<const T *>(w), N, (int)D, chunk, part);
    if (int st = check_launch("weighted_gram")) return st;
    gram_final_kernel<<<8, 256, 0, as_stream(stream)>>>(part, kGramBlocks, (int)D, out);
    return check_launch("weighted_gram_final");
  });
}
