// Selection half of the exact kNN graph (lakde/utils.py:77-116, which ranks
// torch.cdist distances with topk).  The caller computes a block of float64
// squared distances |a|^2 + |b|^2 - 2ab with one library GEMM; this kernel
// turns each row of the block into that point's k nearest neighbours, nearest
// first, equal distances ordered by index:
//
//   1. one CTA per row streams the row once, keeping every value below a
//      running threshold in a shared-memory buffer; when the next chunk could
//      overflow the buffer it is sorted (bitonic, by value then index) and cut
//      to its kc = k + 8 smallest, whose largest becomes the threshold;
//   2. the kc candidates are re-ranked by exact float64 differences
//      sum_d (x_c - x_r)^2 (the GEMM form cancels for close points) and the
//      first k by (exact distance, index) are written.
//
// The point itself is excluded unless include_self (lakde/utils.py:104-105).
#include "common.cuh"

namespace lakde {

// 256 threads per row, or 1,024 when the candidate buffer holds 4,096 or
// more entries (large k: the buffer's sorts dominate, so more threads share
// them; two such CTAs still fit an SM)
constexpr int kKnnThreads = 256, kKnnThreadsLarge = 1024;
constexpr int kKnnChunk = 1024;  // values a CTA scans between buffer checks

// Ascending bitonic sort of n (a power of two) (key, index) pairs in shared
// memory, ties by index; every thread of the CTA takes part.
__device__ __forceinline__ void bitonic_sort(double *key, int32_t *idx, int n) {
  for (int size = 2; size <= n; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      __syncthreads();
      for (int t = threadIdx.x; t < n / 2; t += blockDim.x) {
        const int lo = 2 * t - (t & (stride - 1));
        const int hi = lo + stride;
        const bool up = (lo & size) == 0;
        const double ka = key[lo], kb = key[hi];
        const int32_t ia = idx[lo], ib = idx[hi];
        const bool a_gt_b = ka > kb || (ka == kb && ia > ib);
        if (a_gt_b == up) {
          key[lo] = kb;
          key[hi] = ka;
          idx[lo] = ib;
          idx[hi] = ia;
        }
      }
    }
  }
  __syncthreads();
}

template <typename I, typename O>
__global__ void __launch_bounds__(kKnnThreadsLarge) knn_select_kernel(const double *__restrict__ dist, int64_t N,
                                                                 int64_t row0, const double *__restrict__ X, int D,
                                                                 int include_self, int k, int kc, int cap,
                                                                 I *__restrict__ out_idx, O *__restrict__ out_dist) {
  extern __shared__ double knn_smem[];
  double *key = knn_smem;
  int32_t *idx = reinterpret_cast<int32_t *>(knn_smem + cap);
  __shared__ int cnt;
  __shared__ double thr;
  const int64_t r = blockIdx.x;
  const int64_t self = row0 + r;
  const double *drow = dist + r * N;
  const double inf = __longlong_as_double(0x7ff0000000000000ll);
  if (threadIdx.x == 0) {
    cnt = 0;
    thr = inf;
  }
  __syncthreads();

  // 1. threshold scan
  for (int64_t base = 0; base < N; base += kKnnChunk) {
    // every thread reads the count before any thread adds to it again
    const int c = cnt;
    __syncthreads();
    if (c + kKnnChunk > cap) {
      // pad, sort, keep the kc smallest
      for (int t = c + threadIdx.x; t < cap; t += blockDim.x) {
        key[t] = inf;
        idx[t] = 0x7fffffff;
      }
      bitonic_sort(key, idx, cap);
      if (threadIdx.x == 0) {
        cnt = c < kc ? c : kc;
        thr = c < kc ? inf : key[kc - 1];
      }
      __syncthreads();
    }
    const double t_now = thr;
    for (int u = threadIdx.x; u < kKnnChunk; u += blockDim.x) {
      const int64_t j = base + u;
      if (j < N) {
        double v = drow[j];
        if (v != v || (!include_self && j == self)) v = inf;
        if (v < t_now) {
          const int p = atomicAdd(&cnt, 1);
          key[p] = v;
          idx[p] = (int32_t)j;
        }
      }
    }
    __syncthreads();
  }
  {
    const int c = cnt;
    for (int t = c + threadIdx.x; t < cap; t += blockDim.x) {
      key[t] = inf;
      idx[t] = 0x7fffffff;
    }
    bitonic_sort(key, idx, cap);
  }

  // 2. exact re-ranking of the kc candidates (the rest padded as +inf)
  int n2 = 1;
  while (n2 < kc) n2 <<= 1;
  const double *xr = X + self * D;
  for (int t = threadIdx.x; t < n2; t += blockDim.x) {
    double e = inf;
    int32_t c = 0x7fffffff;
    if (t < kc) {
      c = idx[t];
      if (c >= 0 && c < N && (include_self || c != self)) {
        const double *xc = X + (int64_t)c * D;
        double s = 0.0;
        for (int d = 0; d < D; ++d) {
          const double df = xc[d] - xr[d];
          s = fma(df, df, s);
        }
        e = s;
      } else if (!(c >= 0 && c < N)) {
        c = 0x7fffffff;
      }
    }
    key[t] = e;
    idx[t] = c;
  }
  bitonic_sort(key, idx, n2);
  for (int t = threadIdx.x; t < k; t += blockDim.x) {
    const int32_t c = idx[t];
    out_idx[r * k + t] = (I)(c == 0x7fffffff ? -1 : c);
    if (out_dist) out_dist[r * k + t] = (O)sqrt(key[t]);
  }
}

}  // namespace lakde

using namespace lakde;

extern "C" int lakde_knn_select(const void *dist, int64_t nb, int64_t N, int64_t row0, const void *X, int64_t D,
                                int include_self, int64_t k, int idx_dtype, void *out_idx, int dist_dtype,
                                void *out_dist, void *stream) {
  clear_error();
  if (nb < 0 || N < 1 || D < 1 || row0 < 0 || row0 + nb > N || k < 1 || N > 0x7ffffffeLL) {
    set_error("knn_select: invalid sizes (nb=%lld, N=%lld, D=%lld, row0=%lld, k=%lld)", (long long)nb, (long long)N,
              (long long)D, (long long)row0, (long long)k);
    return LAKDE_EINVAL;
  }
  const int64_t avail = include_self ? N : N - 1;
  if (k > avail) {
    set_error("knn_select: k=%lld exceeds the %lld candidate points", (long long)k, (long long)avail);
    return LAKDE_EINVAL;
  }
  if (nb == 0) return LAKDE_OK;
  if (!dist || !X || !out_idx || (idx_dtype != LAKDE_I32 && idx_dtype != LAKDE_I64) ||
      (out_dist && dist_dtype != LAKDE_F32 && dist_dtype != LAKDE_F64)) {
    set_error("knn_select: null pointer or unsupported dtype");
    return LAKDE_EINVAL;
  }
  const int64_t kc = (k + 8 < avail) ? k + 8 : avail;
  int64_t cap = 2048;
  while (cap < kc + kKnnChunk) cap <<= 1;
  const size_t smem = (size_t)cap * (sizeof(double) + sizeof(int32_t));
  if (smem > 200 * 1024) {
    set_error("knn_select: k=%lld needs %zu bytes of shared memory for its candidates", (long long)k, smem);
    return LAKDE_EUNSUPPORTED;
  }
  if (int st = bind_device("knn_select", {dist, X, out_idx, out_dist})) return st;
  cudaStream_t s = as_stream(stream);
  auto launch = [&](auto ti, auto to) {
    using I = decltype(ti);
    using O = decltype(to);
    auto kern = knn_select_kernel<I, O>;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
      set_error("knn_select: cannot reserve %zu bytes of shared memory", smem);
      return (int)LAKDE_ECUDA;
    }
    const int threads = cap >= 4096 ? kKnnThreadsLarge : kKnnThreads;
    kern<<<(unsigned)nb, threads, smem, s>>>(static_cast<const double *>(dist), N, row0,
                                                 static_cast<const double *>(X), (int)D, include_self, (int)k,
                                                 (int)kc, (int)cap, static_cast<I *>(out_idx),
                                                 static_cast<O *>(out_dist));
    return check_launch("knn_select");
  };
  if (idx_dtype == LAKDE_I32) {
    if (out_dist && dist_dtype == LAKDE_F32) return launch(int32_t(0), float(0));
    return launch(int32_t(0), double(0));
  }
  if (out_dist && dist_dtype == LAKDE_F32) return launch(int64_t(0), float(0));
  return launch(int64_t(0), double(0));
}
