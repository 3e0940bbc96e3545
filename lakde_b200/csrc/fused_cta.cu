// One VI iteration's per-kernel work for 8 < D <= 64, one CTA of 128 threads
// per kernel row (rows visited longest first).  The same quantities as the
// D <= 8 register kernel (lakde_vi_rows):
//
//   1. gather       centred differences (x_m - x_n) of a chunk of <= 128 pairs
//                   into shared memory (fp32), coalesced by point row
//   2. M-step       S_n = sum r (x_m - x_n)(x_m - x_n)^T, each thread a 4x4 block
//                   of the lower triangle (lakde/local_adaptive_kde.py:66-81)
//   3. posterior    A_n = nu_0 a_n / b_n P_n + S_n in FP64 shared memory,
//                   right-looking Cholesky over the 128 threads with the jitter
//                   ladder (lakde/local_adaptive_kde.py:83-96, lakde/linalg_util.py:109-170)
//   4. inverse      L^-1 by right-looking forward substitution (FP64), logdet,
//                   trace ||L^-1 T_n||_F^2, mm_n = nu_n trace, b_n update
//                   (lakde/local_knn_kde.py:220-236)
//   5. E-step       log rho for every pair from the packed W_triu = L^-T in fp32
//                   (lakde/local_adaptive_kde.py:36-44); the differences are
//                   re-gathered only when the row is longer than one chunk.
#include "common.cuh"

namespace lakde {

template <int DP>
struct CtaCfg {
  static constexpr int THREADS = 128;
  static constexpr int CH = 128;               // pairs per chunk
  static constexpr int LDD = DP + 4;           // fp32 row stride of the difference tile
  static constexpr int LDA = DP + 1;           // fp64 row stride of the factor
  static constexpr int NB = DP / 4;            // 4x4 blocks per dimension
  static constexpr int NBLK = NB * (NB + 1) / 2;
  static constexpr int BPT = (NBLK + THREADS - 1) / THREADS;  // blocks per thread
  static constexpr int TS = Tri<float>::size(DP);
  static constexpr size_t off_dlt = 0;
  static constexpr size_t off_A = off_dlt + (size_t)CH * LDD * 4;
  static constexpr size_t off_dinv = off_A + (size_t)DP * LDA * 8;
  static constexpr size_t off_U = off_dinv + (size_t)DP * 8;
  static constexpr size_t off_r = off_U + (size_t)TS * 4;
  static constexpr size_t off_c = off_r + (size_t)CH * 4;
  static constexpr size_t off_xn = off_c + (size_t)CH * 4;
  static constexpr size_t bytes = off_xn + (size_t)LDD * 4;
};

struct CtaArgs {
  const int64_t *rowptr;
  const int32_t *col;
  const int32_t *order;
  const float *r;
  const float *X;
  int64_t npts;
  float nu0;
  const float *P;
  int64_t Pbs;
  const float *Tm;
  int64_t Tbs;
  const float *a;
  float *b;
  float b0;
  float *jitter;
  double eps;
  float *nu_out;
  float *logdet_out;
  float *mm_out;
  int32_t *info;
  float *logrho;
  int64_t N;
  int64_t koff;  // row n is kernel (point) n + koff of X
  int D;
};

// (i, j) of the e-th element of a lower triangle of order m, row-major
__device__ __forceinline__ void tri_decode(int e, int &i, int &j) {
  int ii = (int)((sqrtf(8.f * e + 1.f) - 1.f) * 0.5f);
  while ((ii + 1) * (ii + 2) / 2 <= e) ++ii;
  while (ii * (ii + 1) / 2 > e) --ii;
  i = ii;
  j = e - ii * (ii + 1) / 2;
}

template <int DP>
__device__ __forceinline__ void gather_chunk(const CtaArgs &g, int64_t base, int cnt, float *dlt, float *rv,
                                             int32_t *cidx, const float *xn, bool want_r, int tid, int *bad) {
  using C = CtaCfg<DP>;
  const int D = g.D;
  for (int pp = tid; pp < C::CH; pp += C::THREADS) {
    int32_t c = -1;
    float v = 0.f;
    if (pp < cnt) {
      c = g.col[base + pp];
      if (want_r) v = g.r[base + pp];
      if (c < 0 || c >= g.npts) {
        *bad = 1;
        c = -1;
        v = 0.f;
      }
    }
    cidx[pp] = c;
    rv[pp] = v;
  }
  __syncthreads();
  // one warp per pair row: lanes over dimensions (coalesced)
  const int warp = tid >> 5, lane = tid & 31;
  for (int pp = warp; pp < C::CH; pp += C::THREADS / 32) {
    const int32_t c = cidx[pp];
    for (int d = lane; d < C::LDD; d += 32)
      dlt[pp * C::LDD + d] = (c >= 0 && d < D) ? g.X[(int64_t)c * D + d] - xn[d] : 0.f;
  }
  __syncthreads();
}

template <int DP>
__global__ void __launch_bounds__(128) vi_cta_kernel(CtaArgs g) {
  using C = CtaCfg<DP>;
  extern __shared__ __align__(16) unsigned char smem[];
  float *dlt = reinterpret_cast<float *>(smem + C::off_dlt);
  double *A = reinterpret_cast<double *>(smem + C::off_A);
  double *dinv = reinterpret_cast<double *>(smem + C::off_dinv);
  float *Upk = reinterpret_cast<float *>(smem + C::off_U);
  float *rv = reinterpret_cast<float *>(smem + C::off_r);
  int32_t *cidx = reinterpret_cast<int32_t *>(smem + C::off_c);
  float *xn = reinterpret_cast<float *>(smem + C::off_xn);
  __shared__ int s_bad, s_ok;
  __shared__ double s_red[4];
  __shared__ float s_vsum;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int64_t n = g.order ? (int64_t)g.order[blockIdx.x] : (int64_t)blockIdx.x;
  const int D = g.D;
  const int64_t start = g.rowptr[n], end = g.rowptr[n + 1];
  if (tid == 0) {
    s_bad = end < start ? 1 : 0;
    s_vsum = 0.f;
  }
  for (int d = tid; d < C::LDD; d += C::THREADS) xn[d] = d < D ? g.X[(n + g.koff) * D + d] : 0.f;

  // my 4x4 blocks of the lower triangle
  int bi[C::BPT], bj[C::BPT];
#pragma unroll
  for (int q = 0; q < C::BPT; ++q) {
    const int e = tid + q * C::THREADS;
    if (e < C::NBLK) {
      tri_decode(e, bi[q], bj[q]);
    } else {
      bi[q] = bj[q] = -1;
    }
  }
  float acc[C::BPT][4][4];
#pragma unroll
  for (int q = 0; q < C::BPT; ++q)
#pragma unroll
    for (int p = 0; p < 4; ++p)
#pragma unroll
      for (int s = 0; s < 4; ++s) acc[q][p][s] = 0.f;
  __syncthreads();

  // ----------------------------------------------------------- M-step
  const int64_t len = end > start ? end - start : 0;
  for (int64_t base = start; base < start + len; base += C::CH) {
    const int cnt = (int)((start + len - base) < C::CH ? (start + len - base) : C::CH);
    gather_chunk<DP>(g, base, cnt, dlt, rv, cidx, xn, true, tid, &s_bad);
    if (tid == 0) {
      float s = s_vsum;
      for (int pp = 0; pp < cnt; ++pp) s += rv[pp];
      s_vsum = s;
    }
#pragma unroll
    for (int q = 0; q < C::BPT; ++q) {
      if (bi[q] < 0) continue;
      for (int pp = 0; pp < cnt; ++pp) {
        const float v = rv[pp];
        const float4 a4 = *reinterpret_cast<const float4 *>(dlt + pp * C::LDD + 4 * bi[q]);
        const float4 b4 = *reinterpret_cast<const float4 *>(dlt + pp * C::LDD + 4 * bj[q]);
        const float a[4] = {a4.x, a4.y, a4.z, a4.w};
        const float b[4] = {v * b4.x, v * b4.y, v * b4.z, v * b4.w};
#pragma unroll
        for (int p = 0; p < 4; ++p)
#pragma unroll
          for (int s = 0; s < 4; ++s) acc[q][p][s] = fmaf(a[p], b[s], acc[q][p][s]);
      }
    }
    __syncthreads();
  }
  const float nu = g.nu0 + s_vsum;

  // -------------------------------------------------------- posterior
  const float b_old = g.b[n];
  const float scale = __fmul_rn(g.nu0, __fdiv_rn(g.a[n], b_old));
  const float *P = g.P ? g.P + n * g.Pbs : nullptr;
  float jit = g.jitter[n];
  bool ok = false;
  for (int attempt = 0; attempt <= 32 && !ok; ++attempt) {
    float jt = jit;
    if (attempt > 0) {
      // ladder from zero: eps (2^attempt - 1) after `attempt` rungs
      jt = 0.f;
      for (int k = 0; k < attempt; ++k) jt = __fadd_rn(jt, (float)(g.eps * ldexp(1.0, k)));
    }
    // assemble the lower triangle (padded rows: identity)
    for (int e = tid; e < DP * DP; e += C::THREADS) {
      const int i = e / DP, j = e % DP;
      if (j > i) continue;
      if (i >= D) A[i * C::LDA + j] = (i == j) ? 1.0 : 0.0;
    }
#pragma unroll
    for (int q = 0; q < C::BPT; ++q) {
      if (bi[q] < 0) continue;
#pragma unroll
      for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int s = 0; s < 4; ++s) {
          const int i = 4 * bi[q] + p, j = 4 * bj[q] + s;
          if (j > i || i >= D) continue;
          float v = acc[q][p][s];
          if (P) v = __fadd_rn(__fmul_rn(P[i * D + j], scale), v);
          if (i == j) v = __fadd_rn(v, jt);
          A[i * C::LDA + j] = (double)v;
        }
    }
    if (tid == 0) s_ok = 1;
    __syncthreads();
    for (int k = 0; k < D; ++k) {
      if (tid == 0) {
        const double piv = A[k * C::LDA + k];
        if (!(piv > 0.0)) s_ok = 0;
        const double lkk = sqrt(piv > 0.0 ? piv : 1.0);
        A[k * C::LDA + k] = lkk;
        dinv[k] = 1.0 / lkk;
      }
      __syncthreads();
      const double rk = dinv[k];
      for (int i = k + 1 + tid; i < D; i += C::THREADS) A[i * C::LDA + k] *= rk;
      __syncthreads();
      const int m = D - 1 - k;
      const int T = m * (m + 1) / 2;
      for (int e = tid; e < T; e += C::THREADS) {
        int ii, jj;
        tri_decode(e, ii, jj);
        const int i = k + 1 + ii, j = k + 1 + jj;
        A[i * C::LDA + j] -= A[i * C::LDA + k] * A[j * C::LDA + k];
      }
      __syncthreads();
    }
    ok = s_ok != 0;
    if (ok) jit = jt;
    __syncthreads();  // everyone has read s_ok before the next attempt resets it
  }
  ok = ok && (s_bad == 0);

  // --------------------------------------------- inverse, logdet, trace
  // X = L^-1 stored transposed in the strict upper triangle (A[c][i] = X[i][c],
  // c < i) with the diagonal in dinv; right-looking: after row i of X is final,
  // subtract its contribution from every later row.
  for (int e = tid; e < DP * DP; e += C::THREADS) {
    const int c = e / DP, i = e % DP;
    if (c < i) A[c * C::LDA + i] = 0.0;
  }
  __syncthreads();
  for (int i = 0; i < D; ++i) {
    // row i final: X[i][c] = (delta_ic + acc) / L_ii, acc already in A[c][i]
    for (int c = tid; c < i; c += C::THREADS) A[c * C::LDA + i] *= dinv[i];
    __syncthreads();
    // later rows i2 > i, columns c <= i:  X[i2][c] -= L[i2][i] X[i][c]
    const int rows = D - 1 - i, cols = i + 1;
    for (int e = tid; e < rows * cols; e += C::THREADS) {
      const int i2 = i + 1 + e / cols, c = e % cols;
      const double xic = (c == i) ? dinv[i] : A[c * C::LDA + i];
      A[c * C::LDA + i2] -= A[i2 * C::LDA + i] * xic;
    }
    __syncthreads();
  }
  // logdet_W = 2 sum log W_triu_ii with W_triu_ii = 1 / L_ii rounded to fp32
  double ld = 0.0;
  for (int i = tid; i < D; i += C::THREADS) ld += log((double)(float)dinv[i]);
  // W_triu = X^T (upper): W_triu[r][c] = X[c][r], r <= c -> packed fp32 columns
  for (int e = tid; e < DP * DP; e += C::THREADS) {
    const int r = e / DP, c = e % DP;  // row r, column c of W_triu
    if (r >= Tri<float>::col_len(c)) continue;
    float v = 0.f;
    if (r <= c && c < D) v = (float)(r == c ? dinv[r] : A[r * C::LDA + c]);
    Upk[Tri<float>::col_off(c) + r] = v;
  }
  // trace ||X T_n||_F^2 = sum_{i, a} (sum_k X[i][k] T[k][a])^2 (T_n read once into
  // the difference tile area)
  double tr = 0.0;
  if (g.Tm) {
    float *Ts = dlt;
    const float *Tn = g.Tm + n * g.Tbs;
    for (int e = tid; e < D * D; e += C::THREADS) Ts[e] = Tn[e];
    __syncthreads();
    for (int e = tid; e < D * D; e += C::THREADS) {
      const int i = e / D, a = e % D;
      double s = 0.0;
      for (int k = 0; k <= i; ++k) {
        const double xik = (k == i) ? dinv[i] : A[k * C::LDA + i];
        s += xik * (double)Ts[k * D + a];
      }
      tr += s * s;
    }
  }
  // block reductions of ld and tr
  ld = warp_sum(ld);
  tr = warp_sum(tr);
  __syncthreads();
  if (lane == 0) s_red[warp] = ld;
  __syncthreads();
  const double ld_all = s_red[0] + s_red[1] + s_red[2] + s_red[3];
  __syncthreads();
  if (lane == 0) s_red[warp] = tr;
  __syncthreads();
  const double tr_all = s_red[0] + s_red[1] + s_red[2] + s_red[3];
  const float logdet = (float)(2.0 * ld_all);
  const float mm = nu * (float)tr_all;
  if (tid == 0) {
    const float nanv = NAN;
    g.jitter[n] = jit;
    g.info[n] = ok ? 0 : -1;
    g.nu_out[n] = ok ? nu : nanv;
    g.logdet_out[n] = ok ? logdet : nanv;
    if (g.mm_out) g.mm_out[n] = ok ? mm : nanv;
    if (g.Tm) g.b[n] = ok ? g.b0 + g.nu0 * mm / 2.f : nanv;
  }

  // ------------------------------------------------------------- E-step
  const double e_const = mvdigamma_d(0.5 * (double)nu, D) + D * 0.69314718055994530942 + (double)logdet;
  const float cst = (float)(0.5 * e_const);
  const float expo = -0.5f * nu;
  const bool single = len <= C::CH;
  __syncthreads();
  for (int64_t base = start; base < start + len; base += C::CH) {
    const int cnt = (int)((start + len - base) < C::CH ? (start + len - base) : C::CH);
    if (!single || g.Tm) gather_chunk<DP>(g, base, cnt, dlt, rv, cidx, xn, false, tid, &s_bad);
    for (int pp = tid; pp < cnt; pp += C::THREADS) {
      const int32_t c = cidx[pp];
      float out;
      if (!ok || c < 0) {
        out = NAN;
      } else {
        float delta[DP];
#pragma unroll
        for (int d = 0; d < DP; d += 4) {
          const float4 v = *reinterpret_cast<const float4 *>(dlt + pp * C::LDD + d);
          delta[d] = v.x;
          delta[d + 1] = v.y;
          delta[d + 2] = v.z;
          delta[d + 3] = v.w;
        }
        const float q = quad_tri<float, DP>(Upk, delta);
        out = __fadd_rn(__fmul_rn(q, expo), cst);
        if ((int64_t)c == n + g.koff) out = -INFINITY;
      }
      g.logrho[base + pp] = out;
    }
    __syncthreads();
  }
}

}  // namespace lakde

using namespace lakde;

extern "C" int lakde_vi_cta(int dtype, int64_t N, int64_t D, int64_t npts, const void *rowptr, const void *col,
                            const void *order, const void *r, const void *X, int64_t kernel_offset, double nu_0,
                            const void *P,
                            int64_t P_batch_stride, const void *T, int64_t T_batch_stride, const void *a, void *b,
                            double b_0, void *jitter, double eps, void *nu, void *logdet_W, void *mm,
                            int32_t *info, void *logrho, void *stream) {
  clear_error();
  if (N < 0 || D < 1 || kernel_offset < 0 || npts < N + kernel_offset) {
    set_error("vi_cta: invalid sizes (N=%lld, D=%lld, npts=%lld, kernel_offset=%lld)", (long long)N, (long long)D,
              (long long)npts, (long long)kernel_offset);
    return LAKDE_EINVAL;
  }
  if (N == 0) return LAKDE_OK;
  if (dtype != LAKDE_F32) {
    set_error("vi_cta: float32 values only");
    return LAKDE_EDTYPE;
  }
  if (D <= 8 || D > 64) {
    set_error("vi_cta: D=%lld; the CTA-per-row fused kernel covers 8 < D <= 64", (long long)D);
    return LAKDE_EUNSUPPORTED;
  }
  if (N > 0x7fffffffLL) {
    set_error("vi_cta: N too large");
    return LAKDE_EUNSUPPORTED;
  }
  if (!rowptr || !col || !r || !X || !a || !b || !jitter || !nu || !logdet_W || !info || !logrho) {
    set_error("vi_cta: null pointer");
    return LAKDE_EINVAL;
  }
  if (int st = bind_device("vi_cta", {logrho, rowptr, col, order, r, X, P, T, a, b, jitter, nu, logdet_W, mm, info}))
    return st;
  CtaArgs g;
  g.rowptr = static_cast<const int64_t *>(rowptr);
  g.col = static_cast<const int32_t *>(col);
  g.order = static_cast<const int32_t *>(order);
  g.r = static_cast<const float *>(r);
  g.X = static_cast<const float *>(X);
  g.npts = npts;
  g.nu0 = (float)nu_0;
  g.P = static_cast<const float *>(P);
  g.Pbs = P_batch_stride;
  g.Tm = static_cast<const float *>(T);
  g.Tbs = T_batch_stride;
  g.a = static_cast<const float *>(a);
  g.b = static_cast<float *>(b);
  g.b0 = (float)b_0;
  g.jitter = static_cast<float *>(jitter);
  g.eps = eps;
  g.nu_out = static_cast<float *>(nu);
  g.logdet_out = static_cast<float *>(logdet_W);
  g.mm_out = static_cast<float *>(mm);
  g.info = info;
  g.logrho = static_cast<float *>(logrho);
  g.N = N;
  g.koff = kernel_offset;
  g.D = (int)D;
  auto launch = [&](auto dp) -> int {
    constexpr int DP = decltype(dp)::value;
    using C = CtaCfg<DP>;
    auto kern = vi_cta_kernel<DP>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::bytes);
    if (e != cudaSuccess) {
      set_error("vi_cta: %s", cudaGetErrorString(e));
      return LAKDE_ECUDA;
    }
    kern<<<(unsigned)N, C::THREADS, C::bytes, as_stream(stream)>>>(g);
    return check_launch("vi_cta");
  };
  if (D <= 16) return launch(std::integral_constant<int, 16>{});
  if (D <= 24) return launch(std::integral_constant<int, 24>{});
  if (D <= 32) return launch(std::integral_constant<int, 32>{});
  if (D <= 48) return launch(std::integral_constant<int, 48>{});
  return launch(std::integral_constant<int, 64>{});
}
