// One VI iteration's per-kernel work in a single pass, one thread per kernel
// row, for small D (D <= 8): everything lives in registers.
//
//   M-step     S_n = sum_p r_p (x_m - x_n)(x_m - x_n)^T, nu_n = nu_0 + sum_p r_p
//              (lakde/local_adaptive_kde.py:66-81)
//   posterior  A_n = nu_0 a_n / b_n P_n + S_n, FP64 Cholesky with the jitter
//              ladder (lakde/local_adaptive_kde.py:83-96, lakde/linalg_util.py:109-170)
//   summaries  logdet_W_n = -2 sum log L_ii, trace_n = ||L_n^-1 T_n||_F^2
//              (= ||T_n^T W_triu_n||_F^2), mm_n = nu_n trace_n and the new
//              b_n = b_0 + nu_0 mm_n / 2 (lakde/local_knn_kde.py:220-236)
//   E-step     log rho_p = 0.5 (mvdigamma(nu_n/2) + D log 2 + logdet_W_n)
//              - nu_n / 2 ||L_n^-1 (x_m - x_n)||^2, by forward substitution with
//              L_n (the same quantity as ||W_triu_n^T (x_m - x_n)||^2 with
//              W_triu = L^-T), -inf on the self pair (lakde/local_adaptive_kde.py:36-44)
//
// Rows are visited in a caller-given order (longest first), so the threads of
// a warp carry rows of similar length.
#include "common.cuh"

namespace lakde {

template <typename T>
struct RowArgs {
  const int64_t *rowptr;
  const int32_t *col;
  const int32_t *order;
  const T *r;
  const T *X;
  int64_t npts;
  T nu0;
  const T *P;
  int64_t Pbs;
  const T *Tm;
  int64_t Tbs;
  const T *a;
  T *b;
  T b0;
  T *jitter;
  double eps;
  T *nu_out;
  T *logdet_out;
  T *mm_out;
  int32_t *info;
  T *logrho;
  int64_t N;
  int64_t koff;  // row n is kernel (point) n + koff of X
  int D;
};

__device__ __forceinline__ float f_mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double f_mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float f_add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double f_add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float f_div(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ double f_div(double a, double b) { return __ddiv_rn(a, b); }

template <int DP>
__device__ __forceinline__ constexpr int tix(int i, int j) { return i * (i + 1) / 2 + j; }

// Row m of X (D <= DP, zero padded).  With D == DP and an aligned base the
// rows are DP * 4 or DP * 8 bytes apart and start 16-byte aligned (DP in
// {4, 8}) or 8-byte aligned (DP = 2): vector loads, so a gather of one row per
// thread is one or two load instructions instead of DP.
template <typename T, int DP>
__device__ __forceinline__ void load_row(const T *__restrict__ X, int64_t m, int D, T (&out)[DP]) {
  const uintptr_t base = reinterpret_cast<uintptr_t>(X);
  // rows of 32 bytes (or 64) from a 32-byte aligned base: one 256-bit load
  // per 32 bytes, so a warp's gather of scattered rows touches each row's
  // line once instead of once per 16 bytes
  if constexpr (sizeof(T) * DP >= 32) {
    if (D == DP && (base & 31u) == 0) {
#pragma unroll
      for (int v = 0; v < (int)(sizeof(T) * DP / 32); ++v) {
        const T *p = X + m * DP + v * (32 / (int)sizeof(T));
        if constexpr (sizeof(T) == 4) {
          asm("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                       : "=f"(out[8 * v]), "=f"(out[8 * v + 1]), "=f"(out[8 * v + 2]), "=f"(out[8 * v + 3]),
                         "=f"(out[8 * v + 4]), "=f"(out[8 * v + 5]), "=f"(out[8 * v + 6]), "=f"(out[8 * v + 7])
                       : "l"(p));
        } else {
          asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];"
                       : "=d"(out[4 * v]), "=d"(out[4 * v + 1]), "=d"(out[4 * v + 2]), "=d"(out[4 * v + 3])
                       : "l"(p));
        }
      }
      return;
    }
  }
  if constexpr (sizeof(T) == 4 && DP >= 4) {
    if (D == DP && (base & 15u) == 0) {
      const float4 *p = reinterpret_cast<const float4 *>(X + m * DP);
#pragma unroll
      for (int v = 0; v < DP / 4; ++v) {
        const float4 f = p[v];
        out[4 * v] = f.x;
        out[4 * v + 1] = f.y;
        out[4 * v + 2] = f.z;
        out[4 * v + 3] = f.w;
      }
      return;
    }
  }
  if constexpr (DP >= 2) {
    if (D == DP && (base & (2 * sizeof(T) - 1)) == 0) {
      using V2 = typename std::conditional<sizeof(T) == 4, float2, double2>::type;
      const V2 *p = reinterpret_cast<const V2 *>(X + m * DP);
#pragma unroll
      for (int v = 0; v < DP / 2; ++v) {
        const V2 f = p[v];
        out[2 * v] = f.x;
        out[2 * v + 1] = f.y;
      }
      return;
    }
  }
#pragma unroll
  for (int d = 0; d < DP; ++d) out[d] = d < D ? X[m * D + d] : T(0);
}

// Cholesky of (scale P + S + jit I) in FP64 registers; false if a pivot is
// not positive.  Padded dimensions are the identity.
template <typename T, int DP>
__device__ __forceinline__ bool chol_rows(const T (&S)[DP * (DP + 1) / 2], const T (&Pv)[DP * (DP + 1) / 2],
                                          bool has_p, T scale, T jit, int D, double (&L)[DP * (DP + 1) / 2]) {
#pragma unroll
  for (int i = 0; i < DP; ++i)
#pragma unroll
    for (int j = 0; j <= i; ++j) {
      double v;
      if (i < D) {
        T s = S[tix<DP>(i, j)];
        if (has_p) s = f_add(f_mul(Pv[tix<DP>(i, j)], scale), s);
        if (i == j) s = f_add(s, jit);
        v = (double)s;
      } else {
        v = (i == j) ? 1.0 : 0.0;
      }
      L[tix<DP>(i, j)] = v;
    }
  bool ok = true;
#pragma unroll
  for (int k = 0; k < DP; ++k) {
    const double piv = L[tix<DP>(k, k)];
    ok = ok && (piv > 0.0);
    const double lkk = sqrt(ok ? piv : 1.0);
    const double rk = 1.0 / lkk;
    L[tix<DP>(k, k)] = lkk;
#pragma unroll
    for (int i = k + 1; i < DP; ++i) L[tix<DP>(i, k)] *= rk;
#pragma unroll
    for (int i = k + 1; i < DP; ++i)
#pragma unroll
      for (int j = k + 1; j <= i; ++j) L[tix<DP>(i, j)] -= L[tix<DP>(i, k)] * L[tix<DP>(j, k)];
  }
  return ok;
}

// The per-kernel part of the pass, from the row's scatter S and nu: the
// posterior A = nu_0 a_n / b_n P_n + S + jitter I in FP64 with the jitter
// ladder, logdet_W = -2 sum log L_ii, the trace ||L^-1 T_n||_F^2 by forward
// substitution, mm = nu trace and the b update; writes the per-kernel
// outputs (NaN when the ladder failed or the row had an invalid index) and
// returns whether L holds a factor.
template <typename T, int DP>
__device__ __forceinline__ bool row_posterior(const RowArgs<T> &g, int64_t n, const T (&S)[DP * (DP + 1) / 2], T nu,
                                              bool bad, double (&L)[DP * (DP + 1) / 2], T &logdet) {
  constexpr int TT = DP * (DP + 1) / 2;
  const int D = g.D;
  const T b_old = g.b[n];
  const T scale = f_mul(g.nu0, f_div(g.a[n], b_old));
  // the lower triangle of P_n, row by row (vector loads for D == DP)
  T Pv[TT];
  const bool has_p = g.P != nullptr;
  if (has_p) {
    const T *P = g.P + n * g.Pbs;
#pragma unroll
    for (int i = 0; i < DP; ++i) {
      T row[DP];
      load_row<T, DP>(P, i, D, row);
#pragma unroll
      for (int j = 0; j <= i; ++j) Pv[tix<DP>(i, j)] = i < D ? row[j] : T(0);
    }
  }
  T jit = g.jitter[n];
  bool ok = chol_rows<T, DP>(S, Pv, has_p, scale, jit, D, L);
  if (!ok) {
    T jt = T(0);
    for (int k = 0; k < 32 && !ok; ++k) {
      jt = f_add(jt, (T)(g.eps * ldexp(1.0, k)));
      ok = chol_rows<T, DP>(S, Pv, has_p, scale, jt, D, L);
      if (ok) jit = jt;
    }
  }
  ok = ok && !bad;

  // logdet of W = 2 sum log W_triu_ii, W_triu_ii = 1 / L_ii (in the model dtype)
  double ld = 0.0;
#pragma unroll
  for (int i = 0; i < DP; ++i)
    if (i < D) ld += log((double)(T)(1.0 / L[tix<DP>(i, i)]));
  logdet = (T)(2.0 * ld);

  // trace ||L^-1 T_n||_F^2 by forward substitution of each column of T_n
  // (a column at a time: the whole T_n would not stay in registers)
  double tr = 0.0;
  if (g.Tm) {
    const T *Tn = g.Tm + n * g.Tbs;
#pragma unroll
    for (int a = 0; a < DP; ++a) {
      if (a >= D) continue;
      T tc[DP];
#pragma unroll
      for (int i = 0; i < DP; ++i) tc[i] = i < D ? Tn[i * D + a] : T(0);
      double z[DP];
#pragma unroll
      for (int i = 0; i < DP; ++i) {
        double s = (double)tc[i];
#pragma unroll
        for (int j = 0; j < i; ++j) s -= L[tix<DP>(i, j)] * z[j];
        z[i] = s / L[tix<DP>(i, i)];
        tr += z[i] * z[i];
      }
    }
  }
  const T mm = nu * (T)tr;
  const T nanv = T(NAN);
  g.jitter[n] = jit;
  g.info[n] = ok ? 0 : -1;
  g.nu_out[n] = ok ? nu : nanv;
  g.logdet_out[n] = ok ? logdet : nanv;
  if (g.mm_out) g.mm_out[n] = ok ? mm : nanv;
  if (g.Tm) g.b[n] = ok ? g.b0 + g.nu0 * mm / T(2) : nanv;
  return ok;
}

// float32 with D <= 8: three blocks per SM (168 registers, a few spills to
// L1) hide the pair gathers better than two (0.372 -> 0.329 ms per launch on
// 200,000 rows, K = 50; four blocks spill too much)
template <typename T, int DP>
__global__ void __launch_bounds__(128, (sizeof(T) == 4 && DP == 8) ? 3 : 1) vi_rows_kernel(RowArgs<T> g) {
  constexpr int TT = DP * (DP + 1) / 2;
  const int64_t it = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (it >= g.N) return;
  const int64_t n = g.order ? (int64_t)g.order[it] : it;
  const int D = g.D;
  const int64_t start = g.rowptr[n], end = g.rowptr[n + 1];
  bool bad = end < start;

  T xn[DP];
  load_row<T, DP>(g.X, n + g.koff, D, xn);

  // ---------------------------------------------------------------- M-step
  // pairs in batches of U: the indices, then the point rows of a batch are
  // all loaded before any is used (the gathers of a row overlap); the
  // accumulation order is the pair order
  constexpr int U = 4;
  T S[TT];
#pragma unroll
  for (int e = 0; e < TT; ++e) S[e] = T(0);
  T vsum = T(0);
  for (int64_t p0 = start; p0 < end; p0 += U) {
    int64_t c[U];
    T v[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      c[u] = -1;
      v[u] = T(0);
      if (p0 + u < end) {
        c[u] = g.col[p0 + u];
        v[u] = g.r[p0 + u];
        if (c[u] < 0 || c[u] >= g.npts) {
          bad = true;
          c[u] = -1;
        }
      }
    }
    T dl[U][DP];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      load_row<T, DP>(g.X, c[u] < 0 ? 0 : c[u], D, dl[u]);
#pragma unroll
      for (int d = 0; d < DP; ++d) dl[u][d] = (c[u] >= 0 && d < D) ? dl[u][d] - xn[d] : T(0);
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (c[u] < 0) continue;
#pragma unroll
      for (int i = 0; i < DP; ++i) {
        const T vi = v[u] * dl[u][i];
#pragma unroll
        for (int j = 0; j <= i; ++j) S[tix<DP>(i, j)] = fma(vi, dl[u][j], S[tix<DP>(i, j)]);
      }
      vsum += v[u];
    }
  }
  const T nu = g.nu0 + vsum;
  double L[TT];
  T logdet;
  const bool ok = row_posterior<T, DP>(g, n, S, nu, bad, L, logdet);
  const T nanv = T(NAN);

  // ---------------------------------------------------------------- E-step
  T Lf[TT], rinv[DP];
#pragma unroll
  for (int i = 0; i < DP; ++i) {
#pragma unroll
    for (int j = 0; j < i; ++j) Lf[tix<DP>(i, j)] = (T)L[tix<DP>(i, j)];
    rinv[i] = (T)(1.0 / L[tix<DP>(i, i)]);
  }
  const double e = mvdigamma_d(0.5 * (double)nu, D) + D * 0.69314718055994530942 + (double)logdet;
  const T cst = (T)(0.5 * e);
  const T expo = T(-0.5) * nu;
  for (int64_t p0 = start; p0 < end; p0 += U) {
    int64_t c[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      c[u] = -1;
      if (p0 + u < end) {
        c[u] = g.col[p0 + u];
        if (!ok || c[u] < 0 || c[u] >= g.npts) c[u] = -2;
      }
    }
    T dl[U][DP];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      load_row<T, DP>(g.X, c[u] < 0 ? 0 : c[u], D, dl[u]);
#pragma unroll
      for (int d = 0; d < DP; ++d) dl[u][d] = (c[u] >= 0 && d < D) ? dl[u][d] - xn[d] : T(0);
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (c[u] == -1) continue;  // past the end of the row
      if (c[u] == -2) {
        g.logrho[p0 + u] = nanv;
        continue;
      }
      T y[DP];
      T q = T(0);
#pragma unroll
      for (int i = 0; i < DP; ++i) {
        T s = dl[u][i];
#pragma unroll
        for (int j = 0; j < i; ++j) s = fma(-Lf[tix<DP>(i, j)], y[j], s);
        y[i] = s * rinv[i];
        q = fma(y[i], y[i], q);
      }
      T lr = f_add(f_mul(q, expo), cst);
      if (c[u] == n + g.koff) lr = neg_inf<T>();
      g.logrho[p0 + u] = lr;
    }
  }
}

// The same pass with the pairs of a kernel row dealt to a group of LPR lanes
// and the FP64 posterior one row per lane.  A warp takes 32 consecutive rows
// of the order, 32 / LPR rows at a time in the M- and E-steps: a row's pairs
// go to the group's lanes (pair start + l + LPR k to lane l, so the index,
// responsibility and log rho accesses of a warp are coalesced), in batches of
// B whose gathers are all in flight together.  An xor butterfly sums the
// group's shares of S_n and sum r (every lane ends with the same bits, in a
// fixed order) and lane 0 of the group parks them in the row's slot of the
// warp's shared memory.  Posterior: lane l factorises row l from its slot
// (all 32 lanes on the FP64 work) and parks the factor's pieces in the same
// slot, which the groups read back for the E-step.
template <typename T, int DP>
struct RowSlot {
  static constexpr int TT = DP * (DP + 1) / 2;
  // S (TT), sum r, bad | strictly lower L (TT - DP), 1 / L_ii (DP), c, -nu / 2, ok;
  // an odd stride keeps the lanes' slots on distinct banks
  static constexpr int SIZE = (TT + 4) | 1;
  static constexpr int VSUM = TT, BAD = TT + 1, RINV = TT - DP, CST = TT, EXPO = TT + 1, OK = TT + 2;
};

template <typename T, int DP, int LPR, int B>
__global__ void __launch_bounds__(128, 3) vi_rows_lanes_kernel(RowArgs<T> g) {
  constexpr int TT = DP * (DP + 1) / 2;
  constexpr int GROUPS = 32 / LPR;
  constexpr unsigned FULL = 0xffffffffu;
  using RS = RowSlot<T, DP>;
  __shared__ T park[4][32][RS::SIZE];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, sub = lane & (LPR - 1), grp = lane / LPR;
  const int64_t base = ((int64_t)blockIdx.x * 4 + warp) * 32;
  T(*slot)[RS::SIZE] = park[warp];
  const int D = g.D;
  // each lane loads the setup of one of the warp's rows (row index, pair
  // range, its point row); the groups take their row's from that lane
  int64_t own_n = 0, own_start = 0, own_end = 0;
  if (base + lane < g.N) {
    own_n = g.order ? (int64_t)g.order[base + lane] : base + lane;
    own_start = g.rowptr[own_n];
    own_end = g.rowptr[own_n + 1];
  }
  T own_x[DP];
  load_row<T, DP>(g.X, own_n + g.koff, D, own_x);

  // ---------------------------------------------------------------- M-step
#pragma unroll 1
  for (int pass = 0; pass < LPR; ++pass) {
    const int rl = pass * GROUPS + grp;
    const int64_t n = __shfl_sync(FULL, own_n, rl);
    const int64_t start = __shfl_sync(FULL, own_start, rl);
    int64_t end = __shfl_sync(FULL, own_end, rl);
    T xn[DP];
#pragma unroll
    for (int d = 0; d < DP; ++d) xn[d] = __shfl_sync(FULL, own_x[d], rl);
    int bad = end < start;
    if (bad) end = start;
    T S[TT];
#pragma unroll
    for (int e = 0; e < TT; ++e) S[e] = T(0);
    T vsum = T(0);
    for (int64_t p0 = start + sub; p0 < end; p0 += (int64_t)LPR * B) {
      int32_t c[B];
      T v[B];
#pragma unroll
      for (int k = 0; k < B; ++k) {
        const int64_t p = p0 + (int64_t)LPR * k;
        c[k] = -1;
        v[k] = T(0);
        if (p < end) {
          c[k] = g.col[p];
          v[k] = g.r[p];
          if (c[k] < 0 || c[k] >= g.npts) {
            bad = 1;
            c[k] = -1;
          }
        }
      }
      T dl[B][DP];
#pragma unroll
      for (int k = 0; k < B; ++k) {
        load_row<T, DP>(g.X, c[k] < 0 ? 0 : c[k], D, dl[k]);
#pragma unroll
        for (int d = 0; d < DP; ++d) dl[k][d] = (c[k] >= 0 && d < D) ? dl[k][d] - xn[d] : T(0);
      }
#pragma unroll
      for (int k = 0; k < B; ++k) {
        if (c[k] < 0) continue;
#pragma unroll
        for (int i = 0; i < DP; ++i) {
          const T vi = v[k] * dl[k][i];
#pragma unroll
          for (int j = 0; j <= i; ++j) S[tix<DP>(i, j)] = fma(vi, dl[k][j], S[tix<DP>(i, j)]);
        }
        vsum += v[k];
      }
    }
    // group sums (xor butterfly: the same bits in every lane of the group)
#pragma unroll
    for (int off = LPR / 2; off >= 1; off >>= 1) {
#pragma unroll
      for (int e = 0; e < TT; ++e) S[e] += __shfl_xor_sync(FULL, S[e], off, LPR);
      vsum += __shfl_xor_sync(FULL, vsum, off, LPR);
      bad |= __shfl_xor_sync(FULL, bad, off, LPR);
    }
    if (sub == 0) {
#pragma unroll
      for (int e = 0; e < TT; ++e) slot[rl][e] = S[e];
      slot[rl][RS::VSUM] = vsum;
      slot[rl][RS::BAD] = bad ? T(1) : T(0);
    }
  }
  __syncwarp();

  // ------------------------------------------------------ posterior, a lane per row
  {
    if (base + lane < g.N) {
      const int64_t n = own_n;
      T S[TT];
#pragma unroll
      for (int e = 0; e < TT; ++e) S[e] = slot[lane][e];
      const T nu = g.nu0 + slot[lane][RS::VSUM];
      const bool bad = slot[lane][RS::BAD] != T(0);
      double L[TT];
      T logdet;
      const bool ok = row_posterior<T, DP>(g, n, S, nu, bad, L, logdet);
#pragma unroll
      for (int i = 0; i < DP; ++i) {
#pragma unroll
        for (int j = 0; j < i; ++j) slot[lane][i * (i - 1) / 2 + j] = (T)L[tix<DP>(i, j)];
        slot[lane][RS::RINV + i] = (T)(1.0 / L[tix<DP>(i, i)]);
      }
      const double e = mvdigamma_d(0.5 * (double)nu, D) + D * 0.69314718055994530942 + (double)logdet;
      slot[lane][RS::CST] = (T)(0.5 * e);
      slot[lane][RS::EXPO] = T(-0.5) * nu;
      slot[lane][RS::OK] = ok ? T(1) : T(0);
    }
  }
  __syncwarp();

  // ---------------------------------------------------------------- E-step
  const T nanv = T(NAN);
#pragma unroll 1
  for (int pass = 0; pass < LPR; ++pass) {
    const int rl = pass * GROUPS + grp;
    const int64_t n = __shfl_sync(FULL, own_n, rl);
    const int64_t start = __shfl_sync(FULL, own_start, rl);
    int64_t end = __shfl_sync(FULL, own_end, rl);
    T xn[DP];
#pragma unroll
    for (int d = 0; d < DP; ++d) xn[d] = __shfl_sync(FULL, own_x[d], rl);
    if (base + rl >= g.N) continue;
    if (end < start) end = start;
    T Lf[TT], rinv[DP];
#pragma unroll
    for (int i = 0; i < DP; ++i) {
#pragma unroll
      for (int j = 0; j < i; ++j) Lf[tix<DP>(i, j)] = slot[rl][i * (i - 1) / 2 + j];
      rinv[i] = slot[rl][RS::RINV + i];
    }
    const T cst = slot[rl][RS::CST], expo = slot[rl][RS::EXPO];
    const bool ok = slot[rl][RS::OK] != T(0);
    for (int64_t p0 = start + sub; p0 < end; p0 += (int64_t)LPR * B) {
      int32_t c[B];
#pragma unroll
      for (int k = 0; k < B; ++k) {
        const int64_t p = p0 + (int64_t)LPR * k;
        c[k] = -1;
        if (p < end) {
          c[k] = g.col[p];
          if (!ok || c[k] < 0 || c[k] >= g.npts) c[k] = -2;
        }
      }
      T dl[B][DP];
#pragma unroll
      for (int k = 0; k < B; ++k) {
        load_row<T, DP>(g.X, c[k] < 0 ? 0 : c[k], D, dl[k]);
#pragma unroll
        for (int d = 0; d < DP; ++d) dl[k][d] = (c[k] >= 0 && d < D) ? dl[k][d] - xn[d] : T(0);
      }
#pragma unroll
      for (int k = 0; k < B; ++k) {
        const int64_t p = p0 + (int64_t)LPR * k;
        if (c[k] == -1) continue;  // past the end of the row
        if (c[k] == -2) {
          g.logrho[p] = nanv;
          continue;
        }
        T y[DP];
        T q = T(0);
#pragma unroll
        for (int i = 0; i < DP; ++i) {
          T s2 = dl[k][i];
#pragma unroll
          for (int j = 0; j < i; ++j) s2 = fma(-Lf[tix<DP>(i, j)], y[j], s2);
          y[i] = s2 * rinv[i];
          q = fma(y[i], y[i], q);
        }
        T lr = f_add(f_mul(q, expo), cst);
        if (c[k] == n + g.koff) lr = neg_inf<T>();
        g.logrho[p] = lr;
      }
    }
  }
}

}  // namespace lakde

using namespace lakde;

extern "C" int lakde_vi_rows(int dtype, int64_t N, int64_t D, int64_t npts, const void *rowptr, const void *col,
                             const void *order, const void *r, const void *X, int64_t kernel_offset, double nu_0,
                             const void *P,
                             int64_t P_batch_stride, const void *T, int64_t T_batch_stride, const void *a, void *b,
                             double b_0, void *jitter, double eps, void *nu, void *logdet_W, void *mm,
                             int32_t *info, void *logrho, void *stream) {
  clear_error();
  if (N < 0 || D < 1 || kernel_offset < 0 || npts < N + kernel_offset) {
    set_error("vi_rows: invalid sizes (N=%lld, D=%lld, npts=%lld, kernel_offset=%lld)", (long long)N, (long long)D,
              (long long)npts, (long long)kernel_offset);
    return LAKDE_EINVAL;
  }
  if (N == 0) return LAKDE_OK;
  if (D > 8) {
    set_error("vi_rows: D=%lld; the register-resident fused kernel covers D <= 8", (long long)D);
    return LAKDE_EUNSUPPORTED;
  }
  if (!rowptr || !col || !r || !X || !a || !b || !jitter || !nu || !logdet_W || !info || !logrho) {
    set_error("vi_rows: null pointer");
    return LAKDE_EINVAL;
  }
  if (int st = bind_device("vi_rows", {logrho, rowptr, col, order, r, X, P, T, a, b, jitter, nu, logdet_W, mm, info}))
    return st;
  return dispatch_float(dtype, [&](auto t0) {
    using TT = decltype(t0);
    RowArgs<TT> g;
    g.rowptr = static_cast<const int64_t *>(rowptr);
    g.col = static_cast<const int32_t *>(col);
    g.order = static_cast<const int32_t *>(order);
    g.r = static_cast<const TT *>(r);
    g.X = static_cast<const TT *>(X);
    g.npts = npts;
    g.nu0 = (TT)nu_0;
    g.P = static_cast<const TT *>(P);
    g.Pbs = P_batch_stride;
    g.Tm = static_cast<const TT *>(T);
    g.Tbs = T_batch_stride;
    g.a = static_cast<const TT *>(a);
    g.b = static_cast<TT *>(b);
    g.b0 = (TT)b_0;
    g.jitter = static_cast<TT *>(jitter);
    g.eps = eps;
    g.nu_out = static_cast<TT *>(nu);
    g.logdet_out = static_cast<TT *>(logdet_W);
    g.mm_out = static_cast<TT *>(mm);
    g.info = info;
    g.logrho = static_cast<TT *>(logrho);
    g.N = N;
    g.koff = kernel_offset;
    g.D = (int)D;
    if (tuning(LAKDE_TUNE_VI_ROWS, D) == 1) {
      // a thread per row
      const unsigned blocks = (unsigned)((N + 127) / 128);
      if (D <= 2)
        vi_rows_kernel<TT, 2><<<blocks, 128, 0, as_stream(stream)>>>(g);
      else if (D <= 4)
        vi_rows_kernel<TT, 4><<<blocks, 128, 0, as_stream(stream)>>>(g);
      else
        vi_rows_kernel<TT, 8><<<blocks, 128, 0, as_stream(stream)>>>(g);
      return check_launch("vi_rows");
    }
    // 2 lanes per row for the pairs, a lane per row for the posterior (128
    // rows per 128-thread block; 8 lanes per row measured 10 % slower: more
    // passes of fewer rows each)
    constexpr int LPR = 2, B = sizeof(TT) == 4 ? 4 : 2;
    const int64_t blocks = (N + 127) / 128;
    if (blocks > 0x7fffffffLL) {
      set_error("vi_rows: too many rows");
      return (int)LAKDE_EUNSUPPORTED;
    }
    if (D <= 2)
      vi_rows_lanes_kernel<TT, 2, LPR, B><<<(unsigned)blocks, 128, 0, as_stream(stream)>>>(g);
    else if (D <= 4)
      vi_rows_lanes_kernel<TT, 4, LPR, B><<<(unsigned)blocks, 128, 0, as_stream(stream)>>>(g);
    else
      vi_rows_lanes_kernel<TT, 8, LPR, B><<<(unsigned)blocks, 128, 0, as_stream(stream)>>>(g);
    return check_launch("vi_rows");
  });
}
