// Predictive log density of the Student-t mixture (lakde/local_adaptive_kde.py:200-223):
// a dense kernels x queries sweep fused with the Student-t transform and an
// online logsumexp.  The kernel axis is split into chunks so the grid fills the
// 148 SMs; each (query tile, chunk) CTA leaves a (max, sum) pair per query in a
// caller-provided workspace and a second pass folds the chunks.
#include <mutex>

#include "common.cuh"

namespace lakde {

template <typename T, int DP>
struct PredCfg {
  static constexpr int QT = 128;  // queries per CTA (one per thread)
  static constexpr int KT = DP <= 16 ? 32 : (DP <= 32 ? 16 : 8);
  static constexpr int TS = Tri<T>::size(DP);
  // per-kernel slice: packed factor, centre, log coefficient, (nu+1)/2, padded
  // to a whole 16-byte vector so every slice starts aligned for vector loads
  static constexpr int per_kernel = ((TS + DP + 2 + Tri<T>::V - 1) / Tri<T>::V) * Tri<T>::V;
  static constexpr size_t smem = (size_t)KT * per_kernel * sizeof(T);
};

// Chunk length (kernels per CTA) so that query tiles x chunks ~ 8 CTAs per SM.
static int64_t pred_chunk(int64_t N, int64_t Nq, int kt) {
  const int64_t q_tiles = (Nq + 127) / 128;
  const int64_t target = 148 * 8;
  int64_t nchunks = (target + q_tiles - 1) / q_tiles;
  if (nchunks < 1) nchunks = 1;
  int64_t chunk = (N + nchunks - 1) / nchunks;
  chunk = ((chunk + kt - 1) / kt) * kt;
  if (chunk < kt) chunk = kt;
  return chunk;
}

static int pred_kt(int dtype, int64_t D) {
  int kt = 0;
  dispatch_float(dtype, [&](auto t0) {
    using T = decltype(t0);
    return dispatch_dp(D, [&](auto dp) {
      kt = PredCfg<T, decltype(dp)::value>::KT;
      return 0;
    });
  });
  return kt;
}

// The per-(query, kernel) transcendentals of the predictive density: the
// hardware approximations for float32 (absolute error of log(1 + q) below
// 4e-7, relative error of exp a few ulp near 0; a few 1e-5 nats at most on
// the density after the (nu + 1) / 2 factor), the accurate functions for
// float64.
__device__ __forceinline__ float pred_log1p(float q) { return __logf(1.f + q); }
__device__ __forceinline__ double pred_log1p(double q) { return log1p(q); }
__device__ __forceinline__ float pred_exp(float x) { return __expf(x); }
__device__ __forceinline__ double pred_exp(double x) { return exp(x); }

template <typename T, int DP>
__global__ void __launch_bounds__(128) pred_partial_kernel(const T *__restrict__ X, const T *__restrict__ W,
                                                           const T *__restrict__ nu, const T *__restrict__ lcoef,
                                                           const T *__restrict__ Y, T *__restrict__ ws_m,
                                                           T *__restrict__ ws_s, int64_t N, int64_t Nq, int D,
                                                           int64_t chunk, int64_t q_tiles) {
  using C = PredCfg<T, DP>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *sbase = reinterpret_cast<T *>(smem_raw);
  const int tid = threadIdx.x;
  const int64_t qt = blockIdx.x % q_tiles;
  const int64_t ch = blockIdx.x / q_tiles;
  const int64_t q = qt * C::QT + tid;
  const int64_t n_begin = ch * chunk;
  const int64_t n_end = (n_begin + chunk < N) ? n_begin + chunk : N;

  T y[DP];
#pragma unroll
  for (int d = 0; d < DP; ++d) y[d] = (q < Nq && d < D) ? Y[q * D + d] : T(0);
  T m = neg_inf<T>(), s = T(0);

  for (int64_t n0 = n_begin; n0 < n_end; n0 += C::KT) {
    const int cnt = (int)((n_end - n0) < C::KT ? (n_end - n0) : C::KT);
    __syncthreads();
    for (int k = 0; k < cnt; ++k) {
      T *sk = sbase + k * C::per_kernel;
      const int64_t n = n0 + k;
      load_tri<T, DP>(sk, W + n * (int64_t)D * D, D, 1, D, true, tid, C::QT);
      for (int d = tid; d < DP; d += C::QT) sk[C::TS + d] = d < D ? X[n * D + d] : T(0);
      if (tid == 0) {
        sk[C::TS + DP] = lcoef[n];
        sk[C::TS + DP + 1] = (nu[n] + T(1)) / T(2);
      }
    }
    __syncthreads();
    if (q < Nq) {
      for (int k = 0; k < cnt; ++k) {
        const T *sk = sbase + k * C::per_kernel;
        T delta[DP];
#pragma unroll
        for (int d = 0; d < DP; ++d) delta[d] = y[d] - sk[C::TS + d];
        const T Q = quad_tri<T, DP>(sk, delta);
        const T lp = sk[C::TS + DP] - sk[C::TS + DP + 1] * pred_log1p(Q);
        if (lp == neg_inf<T>()) continue;
        if (lp > m) {
          s = s * pred_exp(m - lp) + T(1);
          m = lp;
        } else {
          s += pred_exp(lp - m);
        }
      }
    }
  }
  if (q < Nq) {
    ws_m[ch * Nq + q] = m;
    ws_s[ch * Nq + q] = s;
  }
}

template <typename T>
__global__ void pred_combine_kernel(const T *__restrict__ ws_m, const T *__restrict__ ws_s, T *__restrict__ out,
                                    int64_t Nq, int64_t nchunks, T log_n) {
  const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (q >= Nq) return;
  T M = neg_inf<T>();
  for (int64_t c = 0; c < nchunks; ++c) M = fmax(M, ws_m[c * Nq + q]);
  T S = T(0);
  if (M != neg_inf<T>())
    for (int64_t c = 0; c < nchunks; ++c) S += ws_s[c * Nq + q] * exp(ws_m[c * Nq + q] - M);
  out[q] = (M == neg_inf<T>()) ? M : (M + log(S)) - log_n;
}

template <typename T>
__global__ void pred_coeff_kernel(const T *__restrict__ nu, const T *__restrict__ logdet, T *__restrict__ out,
                                  int64_t N, int D) {
  const int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (n >= N) return;
  const T a1 = (nu[n] + T(1)) / T(2);
  const T a2 = (nu[n] + T(1) - T(D)) / T(2);
  const T g1 = (T)lgamma((double)a1);
  const T g2 = (T)lgamma((double)a2);
  const double v = (double)g1 - (double)g2 + 0.5 * (double)logdet[n] - 0.5 * D * 1.14472988584940017414;
  out[n] = (T)v;
}

}  // namespace lakde

using namespace lakde;

extern "C" int lakde_pred_coeff(int dtype, int64_t N, int64_t D, const void *nu, const void *logdet_W,
                                void *log_coeff, void *stream) {
  clear_error();
  if (N < 0 || D < 1) {
    set_error("pred_coeff: invalid sizes");
    return LAKDE_EINVAL;
  }
  if (N == 0) return LAKDE_OK;
  if (int st = bind_device("pred_coeff", {log_coeff, nu, logdet_W})) return st;
  return dispatch_float(dtype, [&](auto t0) {
    using T = decltype(t0);
    pred_coeff_kernel<T><<<(unsigned)((N + 255) / 256), 256, 0, as_stream(stream)>>>(
        static_cast<const T *>(nu), static_cast<const T *>(logdet_W), static_cast<T *>(log_coeff), N, (int)D);
    return check_launch("pred_coeff");
  });
}

extern "C" size_t lakde_log_pred_density_workspace(int dtype, int64_t N, int64_t Nq, int64_t D) {
  if (N <= 0 || Nq <= 0 || D < 1 || D > kMaxDim || (dtype != LAKDE_F32 && dtype != LAKDE_F64)) return 0;
  const int kt = pred_kt(dtype, D);
  const int64_t chunk = pred_chunk(N, Nq, kt);
  const int64_t nchunks = (N + chunk - 1) / chunk;
  const size_t es = dtype == LAKDE_F32 ? 4 : 8;
  return (size_t)(2 * nchunks * Nq) * es;
}

// The partial and fold launches of the predictive density over the (max, sum)
// scratch `ws` (lakde_log_pred_density_workspace bytes), shared by the
// workspace and the allocation-free entry points.
static int launch_pred(const char *what, int dtype, int64_t N, int64_t Nq, int64_t D, const void *X,
                       const void *W_triu, const void *nu, const void *log_coeff, const void *Y, void *out, void *ws,
                       void *stream) {
  return dispatch_float(dtype, [&](auto t0) {
    using T = decltype(t0);
    return dispatch_dp(D, [&](auto dp) {
      constexpr int DP = decltype(dp)::value;
      using C = PredCfg<T, DP>;
      const int64_t chunk = pred_chunk(N, Nq, C::KT);
      const int64_t nchunks = (N + chunk - 1) / chunk;
      const int64_t q_tiles = (Nq + C::QT - 1) / C::QT;
      if (q_tiles * nchunks > 0x7fffffffLL) {
        set_error("%s: grid too large", what);
        return (int)LAKDE_EUNSUPPORTED;
      }
      auto kern = pred_partial_kernel<T, DP>;
      if (C::smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::smem);
        if (e != cudaSuccess) {
          set_error("%s: %s", what, cudaGetErrorString(e));
          return (int)LAKDE_ECUDA;
        }
      }
      T *ws_m = static_cast<T *>(ws);
      T *ws_s = ws_m + nchunks * Nq;
      kern<<<(unsigned)(q_tiles * nchunks), C::QT, C::smem, as_stream(stream)>>>(
          static_cast<const T *>(X), static_cast<const T *>(W_triu), static_cast<const T *>(nu),
          static_cast<const T *>(log_coeff), static_cast<const T *>(Y), ws_m, ws_s, N, Nq, (int)D, chunk, q_tiles);
      if (int st = check_launch(what)) return st;
      pred_combine_kernel<T><<<(unsigned)((Nq + 255) / 256), 256, 0, as_stream(stream)>>>(
          ws_m, ws_s, static_cast<T *>(out), Nq, nchunks, (T)log((double)N));
      return check_launch(what);
    });
  });
}

extern "C" int lakde_log_pred_density(int dtype, int64_t N, int64_t Nq, int64_t D, const void *X, const void *W_triu,
                                      const void *nu, const void *log_coeff, const void *Y, void *out,
                                      void *workspace, size_t workspace_bytes, void *stream) {
  clear_error();
  if (N < 1 || Nq < 0 || D < 1) {
    set_error("log_pred_density: invalid sizes (N=%lld, Nq=%lld, D=%lld)", (long long)N, (long long)Nq,
              (long long)D);
    return LAKDE_EINVAL;
  }
  if (Nq == 0) return LAKDE_OK;
  const size_t need = lakde_log_pred_density_workspace(dtype, N, Nq, D);
  if (need == 0) {
    set_error("log_pred_density: unsupported dtype %d or D=%lld", dtype, (long long)D);
    return LAKDE_EUNSUPPORTED;
  }
  if (!workspace || workspace_bytes < need) {
    set_error("log_pred_density: workspace of %zu bytes needed, %zu given", need, workspace_bytes);
    return LAKDE_EINVAL;
  }
  if (!X || !W_triu || !nu || !log_coeff || !Y || !out) {
    set_error("log_pred_density: null pointer");
    return LAKDE_EINVAL;
  }
  if (int st = bind_device("log_pred_density", {out, X, W_triu, nu, log_coeff, Y, workspace})) return st;
  return launch_pred("log_pred_density", dtype, N, Nq, D, X, W_triu, nu, log_coeff, Y, out, workspace, stream);
}

// ---------------------------------------------------------------------------
// Allocation-free variant.  Some callers cannot call cudaMalloc: hosts that own
// all device memory themselves (a framework's caching allocator, a plugin
// sandbox) or that forbid device allocation once they are running.  For them
// the (max, sum) partials live in this file-scope device array instead of a
// caller workspace.  It is 16 MiB; every GPU that loads the library holds it
// until the process exits.  All calls share it, and it keeps the contents of the
// last call: every slot a call reads is written earlier in that same call, so
// nothing needs clearing, but calls that overlap on the GPU (concurrent
// streams, or several host threads) race on it.
// ---------------------------------------------------------------------------
namespace lakde {

constexpr size_t kNoAllocScratchBytes = 16u << 20;
static __device__ __align__(256) unsigned char g_pred_scratch[kNoAllocScratchBytes];

// Device address of g_pred_scratch per device, resolved on the first call that
// runs on that device (with the device current) and kept for the life of the
// process.  A cudaDeviceReset destroys the array with the context, so the
// address is not valid across one (nor is any other device pointer).
constexpr int kMaxDevices = 128;
static void *g_pred_scratch_ptr[kMaxDevices];
static std::mutex g_pred_scratch_mu;

static int pred_scratch_address(void **out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    set_error("log_pred_density_noalloc: cudaGetDevice failed: %s", cudaGetErrorString(e));
    return LAKDE_ECUDA;
  }
  if (dev < 0 || dev >= kMaxDevices) {
    set_error("log_pred_density_noalloc: device index %d is beyond the %d devices this entry point serves", dev,
              kMaxDevices);
    return LAKDE_EUNSUPPORTED;
  }
  std::lock_guard<std::mutex> lock(g_pred_scratch_mu);
  if (!g_pred_scratch_ptr[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_pred_scratch);
    if (e != cudaSuccess || !p) {
      set_error("log_pred_density_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
      return LAKDE_ECUDA;
    }
    g_pred_scratch_ptr[dev] = p;
  }
  *out = g_pred_scratch_ptr[dev];
  return LAKDE_OK;
}

}  // namespace lakde

extern "C" int lakde_log_pred_density_noalloc(int dtype, int64_t N, int64_t Nq, int64_t D, const void *X,
                                              const void *W_triu, const void *nu, const void *log_coeff,
                                              const void *Y, void *out, void *stream) {
  clear_error();
  if (N < 1 || Nq < 0 || D < 1) {
    set_error("log_pred_density_noalloc: invalid sizes (N=%lld, Nq=%lld, D=%lld)", (long long)N, (long long)Nq,
              (long long)D);
    return LAKDE_EINVAL;
  }
  if (Nq == 0) return LAKDE_OK;
  const size_t need = lakde_log_pred_density_workspace(dtype, N, Nq, D);
  if (need == 0) {
    set_error("log_pred_density_noalloc: unsupported dtype %d or D=%lld", dtype, (long long)D);
    return LAKDE_EUNSUPPORTED;
  }
  if (need > kNoAllocScratchBytes) {
    set_error("log_pred_density_noalloc: %lld queries x %lld kernels need %zu bytes of scratch, more than the "
              "built-in %zu bytes; split the queries into smaller batches",
              (long long)Nq, (long long)N, need, kNoAllocScratchBytes);
    return LAKDE_EINVAL;
  }
  if (!X || !W_triu || !nu || !log_coeff || !Y || !out) {
    set_error("log_pred_density_noalloc: null pointer");
    return LAKDE_EINVAL;
  }
  if (int st = bind_device("log_pred_density_noalloc", {out, X, W_triu, nu, log_coeff, Y})) return st;
  void *scratch = nullptr;
  if (int st = pred_scratch_address(&scratch)) return st;
  return launch_pred("log_pred_density_noalloc", dtype, N, Nq, D, X, W_triu, nu, log_coeff, Y, out, scratch, stream);
}
