// Batched posterior factorisation in FP64:
//   A_n = nu_0 E[tau_n] P_n + S_n  ->  L_n = chol(A_n + jitter_n I)  ->  W_triu_n = L_n^-T
// with the per-matrix jitter ladder of lakde/linalg_util.py:109-170 run on the
// device (no host round trip per failed matrix), plus logdet_W and the trace
// term ||T_n^T W_triu_n||_F^2 (lakde/linalg_util.py:30-37).
//
// D <= 8: one thread per matrix, everything in registers.
// D in (8, 64]: one warp per matrix on the FP64 tensor cores (mma.sync
// m8n8k4 f64): blocked right-looking Cholesky over 8 x 8 lower tiles in shared
// memory, in-place blocked triangular inverse, trace by tile products
// (factor_dmma.cuh).
#include "common.cuh"
#include "factor_dmma.cuh"

namespace lakde {

template <typename T>
struct FactorArgs {
  const T *S;
  const T *P;
  int64_t Pbs;
  const T *nu0;
  const T *a;
  const T *b;
  T *jitter;
  double eps;
  T *W;
  T *L;
  T *logdet;
  int32_t *info;
  const T *Tm;
  int64_t Tbs;
  T *trace;
  int64_t N;
  int D;
};

// Round-to-nearest arithmetic without contraction, to reproduce the rounding of
// the reference's separate tensor ops (scale * P, + S, + jitter).
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float div_rn(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ double div_rn(double a, double b) { return __ddiv_rn(a, b); }

template <typename T>
__device__ __forceinline__ T posterior_scale(const FactorArgs<T> &g, int64_t n) {
  if (g.a && g.b) return mul_rn(g.nu0 ? g.nu0[0] : T(1), div_rn(g.a[n], g.b[n]));
  return T(1);
}

// A_ij (lower part) of matrix n in the model dtype, jitter on the diagonal.
template <typename T>
__device__ __forceinline__ double assembled(const FactorArgs<T> &g, int64_t n, T scale, int i, int j, T jit) {
  const int D = g.D;
  T v = g.S[n * (int64_t)D * D + i * D + j];
  if (g.P) v = add_rn(mul_rn(g.P[n * g.Pbs + i * D + j], scale), v);
  if (i == j) v = add_rn(v, jit);
  return (double)v;
}

// ----------------------------- thread per matrix ---------------------------
template <int DP>
__device__ __forceinline__ int tri_idx(int i, int j) { return i * (i + 1) / 2 + j; }

template <typename T, int DP>
__device__ __forceinline__ bool chol_regs(const FactorArgs<T> &g, int64_t n, T scale, T jit,
                                          double (&L)[DP * (DP + 1) / 2]) {
  const int D = g.D;
#pragma unroll
  for (int i = 0; i < DP; ++i)
#pragma unroll
    for (int j = 0; j <= i; ++j) L[tri_idx<DP>(i, j)] = (i < D) ? assembled(g, n, scale, i, j, jit) : (i == j ? 1.0 : 0.0);
  bool ok = true;
#pragma unroll
  for (int k = 0; k < DP; ++k) {
    const double piv = L[tri_idx<DP>(k, k)];
    ok = ok && (piv > 0.0);
    const double lkk = sqrt(ok ? piv : 1.0);
    const double r = 1.0 / lkk;
    L[tri_idx<DP>(k, k)] = lkk;
#pragma unroll
    for (int i = k + 1; i < DP; ++i) L[tri_idx<DP>(i, k)] *= r;
#pragma unroll
    for (int i = k + 1; i < DP; ++i)
#pragma unroll
      for (int j = k + 1; j <= i; ++j) L[tri_idx<DP>(i, j)] -= L[tri_idx<DP>(i, k)] * L[tri_idx<DP>(j, k)];
  }
  return ok;
}

template <typename T, int DP>
__global__ void __launch_bounds__(128) factor_thread_kernel(FactorArgs<T> g) {
  constexpr int TT = DP * (DP + 1) / 2;
  const int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (n >= g.N) return;
  const int D = g.D;
  const T scale = posterior_scale(g, n);
  T jit = g.jitter[n];
  double L[TT];
  bool ok = chol_regs<T, DP>(g, n, scale, jit, L);
  if (!ok) {
    T jt = T(0);
    for (int k = 0; k < 32 && !ok; ++k) {
      jt = add_rn(jt, (T)(g.eps * ldexp(1.0, k)));
      ok = chol_regs<T, DP>(g, n, scale, jt, L);
      if (ok) jit = jt;
    }
  }
  g.jitter[n] = jit;
  g.info[n] = ok ? 0 : -1;
  // inverse of L (lower), column by column
  double Li[TT];
#pragma unroll
  for (int c = 0; c < DP; ++c) {
    Li[tri_idx<DP>(c, c)] = 1.0 / L[tri_idx<DP>(c, c)];
#pragma unroll
    for (int i = c + 1; i < DP; ++i) {
      double s = 0.0;
#pragma unroll
      for (int k = c; k < i; ++k) s += L[tri_idx<DP>(i, k)] * Li[tri_idx<DP>(k, c)];
      Li[tri_idx<DP>(i, c)] = -s / L[tri_idx<DP>(i, i)];
    }
  }
  const T nanv = T(NAN);
  T *W = g.W + n * (int64_t)D * D;
  double ld = 0.0;
#pragma unroll
  for (int r = 0; r < DP; ++r) {
    if (r >= D) continue;
#pragma unroll
    for (int c = 0; c < DP; ++c) {
      if (c >= D) continue;
      const double u = (r <= c) ? Li[tri_idx<DP>(c, r)] : 0.0;
      W[r * D + c] = ok ? (T)u : nanv;
    }
    ld += log((double)(T)Li[tri_idx<DP>(r, r)]);
  }
  g.logdet[n] = ok ? (T)(2.0 * ld) : nanv;
  if (g.L) {
    T *Lo = g.L + n * (int64_t)D * D;
#pragma unroll
    for (int r = 0; r < DP; ++r) {
      if (r >= D) continue;
#pragma unroll
      for (int c = 0; c < DP; ++c)
        if (c < D) Lo[r * D + c] = ok ? (T)((r >= c) ? L[tri_idx<DP>(r, c)] : 0.0) : nanv;
    }
  }
  if (g.Tm) {
    const T *Tm = g.Tm + n * g.Tbs;
    double acc = 0.0;
    for (int a = 0; a < D; ++a) {
#pragma unroll
      for (int bcol = 0; bcol < DP; ++bcol) {
        if (bcol >= D) continue;
        double s = 0.0;
#pragma unroll
        for (int k = 0; k <= bcol; ++k) s += (double)Tm[k * D + a] * Li[tri_idx<DP>(bcol, k)];
        acc += s * s;
      }
    }
    g.trace[n] = ok ? (T)acc : nanv;
  }
}

// ------------------------- warp per matrix, FP64 tensor cores --------------
template <int DP>
struct DmmaCfg {
  static constexpr int NT = DP / 8;
  static constexpr int NTILE = NT * (NT + 1) / 2;
  static constexpr int WPB = DP >= 48 ? 2 : 4;
  static constexpr int per_warp = NTILE * 64 + 64 + DP + NT * 64;  // tiles, scratch, diag(L), T column block
  static constexpr size_t smem = (size_t)WPB * per_warp * sizeof(double);
};

template <typename T, int DP>
__global__ void __launch_bounds__(128) factor_dmma_kernel(FactorArgs<T> g) {
  using C = DmmaCfg<DP>;
  constexpr int NT = C::NT;
  extern __shared__ double smem_d[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t n = (int64_t)blockIdx.x * C::WPB + warp;
  if (n >= g.N) return;
  double *M = smem_d + warp * C::per_warp;
  double *scratch = M + C::NTILE * 64;
  double *ldiag = scratch + 64;
  double *tcol = ldiag + DP;  // one 8-column block of T_n, NT tiles
  const int D = g.D;
  const T scale = posterior_scale(g, n);
  T jit = g.jitter[n];
  T *lout = g.L ? g.L + n * (int64_t)D * D : nullptr;
  bool ok = false;
  for (int attempt = 0; attempt <= 32 && !ok; ++attempt) {
    T jt = jit;
    if (attempt > 0) {
      jt = T(0);
      for (int k = 0; k < attempt; ++k) jt = add_rn(jt, (T)(g.eps * ldexp(1.0, k)));
    }
    for (int e = lane; e < DP * DP; e += 32) {
      const int i = e / DP, j = e % DP;
      if (j > i) continue;
      const double v = (i < D) ? assembled(g, n, scale, i, j, jt) : (i == j ? 1.0 : 0.0);
      M[dmma::tix(i >> 3, j >> 3) + (i & 7) * 8 + (j & 7)] = v;
    }
    __syncwarp();
    ok = dmma::chol_blocked<T>(M, scratch, ldiag, NT, lane, lout, D);
    if (ok) jit = jt;
    __syncwarp();
  }
  if (lane == 0) {
    g.jitter[n] = jit;
    g.info[n] = ok ? 0 : -1;
  }
  const T nanv = T(NAN);
  T *W = g.W + n * (int64_t)D * D;
  if (!ok) {
    for (int e = lane; e < D * D; e += 32) {
      W[e] = nanv;
      if (lout) lout[e] = nanv;
    }
    if (lane == 0) {
      g.logdet[n] = nanv;
      if (g.Tm) g.trace[n] = nanv;
    }
    return;
  }
  if (lout) {
    // the factor's strictly upper blocks are not touched by the tile loops
    for (int e = lane; e < D * D; e += 32) {
      const int r = e / D, c = e % D;
      if ((c >> 3) > (r >> 3)) lout[e] = T(0);
    }
  }
  dmma::trtri_blocked(M, scratch, NT, lane);
  // W_triu = X^T (upper): W[r][c] = X[c][r], r <= c
  for (int e = lane; e < D * D; e += 32) {
    const int r = e / D, c = e % D;
    const double v = (r <= c) ? M[dmma::tix(c >> 3, r >> 3) + (c & 7) * 8 + (r & 7)] : 0.0;
    W[e] = (T)v;
  }
  double ld = 0.0;
  for (int i = lane; i < D; i += 32) ld += log((double)(T)(1.0 / ldiag[i]));
  ld = warp_sum(ld);
  if (lane == 0) g.logdet[n] = (T)(2.0 * ld);
  if (g.Tm) {
    // ||X T_n||_F^2 with X lower: (X T)_IA = sum_{K <= I} X_IK T_KA.  Each
    // 8-column block A of T_n is staged in shared memory (coalesced rows) and
    // its all-zero 8 x 8 tiles (the upper part of a triangular T) are skipped.
    const T *Tn = g.Tm + n * g.Tbs;
    double acc = 0.0;
    for (int Ac = 0; Ac < NT; ++Ac) {
      __syncwarp();
      for (int e = lane; e < NT * 64; e += 32) {
        const int row = e >> 3, col = 8 * Ac + (e & 7);
        tcol[e] = (row < D && col < D) ? (double)Tn[row * D + col] : 0.0;
      }
      __syncwarp();
      unsigned nonzero = 0;  // bit K: tile K of this column block has a non-zero
      for (int K = 0; K < NT; ++K) {
        const bool nz = tcol[K * 64 + lane] != 0.0 || tcol[K * 64 + 32 + lane] != 0.0;
        if (__any_sync(0xffffffffu, nz)) nonzero |= 1u << K;
      }
      for (int I = 0; I < NT; ++I) {
        double c0 = 0.0, c1 = 0.0;
        for (int K = 0; K <= I; ++K) {
          if (!((nonzero >> K) & 1u)) continue;
          const double *x = M + dmma::tix(I, K);
          const double *tk = tcol + K * 64;
#pragma unroll
          for (int s = 0; s < 2; ++s) dmma::mma(c0, c1, dmma::afrag(x, s, lane), dmma::bfrag(tk, s, lane));
        }
        acc += c0 * c0 + c1 * c1;
      }
    }
    acc = warp_sum(acc);
    if (lane == 0) g.trace[n] = (T)acc;
  }
}

}  // namespace lakde

using namespace lakde;

extern "C" int lakde_posterior_factor(int dtype, int64_t N, int64_t D, const void *S, const void *P,
                                      int64_t P_batch_stride, const void *nu_0, const void *a, const void *b,
                                      void *jitter, double eps, void *W_triu, void *L, void *logdet_W,
                                      int32_t *info, const void *T, int64_t T_batch_stride, void *trace,
                                      void *stream) {
  clear_error();
  if (N < 0 || D < 1) {
    set_error("posterior_factor: invalid sizes (N=%lld, D=%lld)", (long long)N, (long long)D);
    return LAKDE_EINVAL;
  }
  if (N == 0) return LAKDE_OK;
  if (!S || !jitter || !W_triu || !logdet_W || !info || (T && !trace) || ((a == nullptr) != (b == nullptr))) {
    set_error("posterior_factor: missing buffer");
    return LAKDE_EINVAL;
  }
  if (N > 0x7fffffffLL) {
    set_error("posterior_factor: N too large");
    return LAKDE_EUNSUPPORTED;
  }
  if (int st = bind_device("posterior_factor", {W_triu, S, P, nu_0, a, b, jitter, L, logdet_W, info, T, trace}))
    return st;
  return dispatch_float(dtype, [&](auto t0) {
    using TT = decltype(t0);
    FactorArgs<TT> g;
    g.S = static_cast<const TT *>(S);
    g.P = static_cast<const TT *>(P);
    g.Pbs = P_batch_stride;
    g.nu0 = static_cast<const TT *>(nu_0);
    g.a = static_cast<const TT *>(a);
    g.b = static_cast<const TT *>(b);
    g.jitter = static_cast<TT *>(jitter);
    g.eps = eps;
    g.W = static_cast<TT *>(W_triu);
    g.L = static_cast<TT *>(L);
    g.logdet = static_cast<TT *>(logdet_W);
    g.info = info;
    g.Tm = static_cast<const TT *>(T);
    g.Tbs = T_batch_stride;
    g.trace = static_cast<TT *>(trace);
    g.N = N;
    g.D = (int)D;
    return dispatch_dp(D, [&](auto dp) {
      constexpr int DP = decltype(dp)::value;
      if constexpr (DP <= 8) {
        factor_thread_kernel<TT, DP><<<(unsigned)((N + 127) / 128), 128, 0, as_stream(stream)>>>(g);
      } else {
        using C = DmmaCfg<DP>;
        auto kern = factor_dmma_kernel<TT, DP>;
        if (C::smem > 48 * 1024) {
          cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::smem);
          if (e != cudaSuccess) {
            set_error("posterior_factor: %s", cudaGetErrorString(e));
            return (int)LAKDE_ECUDA;
          }
        }
        kern<<<(unsigned)((N + C::WPB - 1) / C::WPB), 32 * C::WPB, C::smem, as_stream(stream)>>>(g);
      }
      return check_launch("posterior_factor");
    });
  });
}
