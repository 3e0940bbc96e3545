// Weighted Gram sum of the hierarchical model's shared-precision update in
// FP64 (lakde/local_hierarchical_kde.py:293-297):
//   out = sum_n w_n W_triu_n W_triu_n^T        (D x D, symmetric)
// straight from the float32 (or float64) factors, without a float64 copy of
// all of them.  Each CTA walks a contiguous chunk of kernels, stages W_triu_n
// transposed in shared memory (column j of W as a row, zero below the
// diagonal), and each thread accumulates one 4 x 4 block of the lower
// triangle in FP64 registers: per column j two 16-byte loads of its block's
// rows and two of its block's columns feed 16 FMAs.  The per-CTA partials are
// summed in a fixed order by the final kernel, so the result does not depend
// on scheduling.
#include "common.cuh"

namespace lakde {

constexpr int kGramBlocks = 592;
constexpr int kGramThreads = 160;  // >= the 136 lower 4 x 4 blocks at D = 64

template <typename T>
__global__ void __launch_bounds__(kGramThreads) gram_partial_kernel(const T *__restrict__ W, const T *__restrict__ w,
                                                                   int64_t N, int D, int64_t chunk,
                                                                   double *__restrict__ partials) {
  extern __shared__ double sWt[];  // [DP][DP]: sWt[j * DP + i] = W[i][j] for j >= i, else 0
  const int DP = (D + 3) & ~3, nb = DP / 4;
  const int tri = D * (D + 1) / 2;
  const int tid = threadIdx.x;
  int bi = 0;
  while ((bi + 1) * (bi + 2) / 2 <= tid) ++bi;
  const int bk = tid - bi * (bi + 1) / 2;
  const bool active = bi < nb;
  double acc[4][4];
#pragma unroll
  for (int x = 0; x < 4; ++x)
#pragma unroll
    for (int y = 0; y < 4; ++y) acc[x][y] = 0.0;
  const int64_t n0 = (int64_t)blockIdx.x * chunk;
  const int64_t n1 = (n0 + chunk < N) ? n0 + chunk : N;
  for (int64_t n = n0; n < n1; ++n) {
    const T *Wn = W + n * (int64_t)D * D;
    __syncthreads();
    // coalesced over the row-major W_triu_n, stored transposed
    for (int e = tid; e < DP * DP; e += kGramThreads) {
      const int i = e / DP, j = e % DP;
      sWt[j * DP + i] = (i < D && j < D && j >= i) ? (double)Wn[i * D + j] : 0.0;
    }
    __syncthreads();
    if (!active) continue;
    const double wn = (double)w[n];
    double t[4][4];
#pragma unroll
    for (int x = 0; x < 4; ++x)
#pragma unroll
      for (int y = 0; y < 4; ++y) t[x][y] = 0.0;
    // (W W^T)_ik = sum_j W_ij W_kj over j >= max(i, k) >= 4 bk
    for (int j = 4 * bk; j < DP; ++j) {
      const double *col = sWt + j * DP;
      const double2 a01 = *reinterpret_cast<const double2 *>(col + 4 * bi);
      const double2 a23 = *reinterpret_cast<const double2 *>(col + 4 * bi + 2);
      const double2 b01 = *reinterpret_cast<const double2 *>(col + 4 * bk);
      const double2 b23 = *reinterpret_cast<const double2 *>(col + 4 * bk + 2);
      const double a[4] = {a01.x, a01.y, a23.x, a23.y}, b[4] = {b01.x, b01.y, b23.x, b23.y};
#pragma unroll
      for (int x = 0; x < 4; ++x)
#pragma unroll
        for (int y = 0; y < 4; ++y) t[x][y] = fma(a[x], b[y], t[x][y]);
    }
#pragma unroll
    for (int x = 0; x < 4; ++x)
#pragma unroll
      for (int y = 0; y < 4; ++y) acc[x][y] = fma(wn, t[x][y], acc[x][y]);
  }
  if (!active) return;
#pragma unroll
  for (int x = 0; x < 4; ++x)
#pragma unroll
    for (int y = 0; y < 4; ++y) {
      const int i = 4 * bi + x, k = 4 * bk + y;
      if (i < D && k <= i) partials[(int64_t)blockIdx.x * tri + i * (i + 1) / 2 + k] = acc[x][y];
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
    const int DP = (int)((D + 3) & ~3);
    gram_partial_kernel<T><<<kGramBlocks, kGramThreads, (size_t)DP * DP * sizeof(double), as_stream(stream)>>>(
        static_cast<const T *>(W_triu), static_cast<const T *>(w), N, (int)D, chunk, part);
    if (int st = check_launch("weighted_gram")) return st;
    gram_final_kernel<<<8, 256, 0, as_stream(stream)>>>(part, kGramBlocks, (int)D, out);
    return check_launch("weighted_gram_final");
  });
}
