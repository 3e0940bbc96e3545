// Batched posterior factorisation in FP64:
//   A_n = nu_0 E[tau_n] P_n + S_n  ->  L_n = chol(A_n + jitter_n I)  ->  W_triu_n = L_n^-T
// with the per-matrix jitter ladder of lakde/linalg_util.py:109-170 run on the
// device (no host round trip per failed matrix), plus logdet_W and the trace
// term ||T_n^T W_triu_n||_F^2 (lakde/linalg_util.py:30-37).
//
// D <= 8: one thread per matrix, everything in registers.
// D in (8, 64]: one warp per matrix on the FP64 tensor cores (mma.sync
// m8n8k4 f64): blocked right-looking Cholesky over 8 x 8 lower tiles in shared
// memory with the triangular inverse formed in the same sweep, trace by tile
// products (factor_dmma.cuh).
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
  int T_lower;
  T *trace;
  // tiled inputs (float32, 8 < D <= 64): per matrix, tile t of the lower
  // 8 x 8 tiles of S then of P (SP, 128 floats per tile) and of T (Tt, 64)
  const float *SP;
  const float *Tt;
  float *Xt;  // optional output: X = L^-1 (= W_triu^T) as lower tiles, 64 floats per tile
  // optional output: X = L^-1 (= W_triu^T) as the W cores of the tensor-core
  // E-step's B operand, 64 floats per tile (layout at lakde_pack_w_cores)
  float *Wc;
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
        for (int k = 0; k <= bcol; ++k) {
          const double tka = (g.T_lower && a > k) ? 0.0 : (double)Tm[k * D + a];
          s += tka * Li[tri_idx<DP>(bcol, k)];
        }
        acc += s * s;
      }
    }
    g.trace[n] = ok ? (T)acc : nanv;
  }
}

// ------------------------- warp per matrix, FP64 tensor cores --------------
template <int DP, bool LEAN = false>
struct DmmaCfg {
  static constexpr int NT = DP / 8;
  static constexpr int NTILE = NT * (NT + 1) / 2;
  // LEAN: no per-matrix T_n staged (the trace reads its tiles from global
  // memory) and no L output: ~19 KB per warp at DP = 64, one warp per block,
  // 11 blocks per SM (registers capped to fit)
  static constexpr int WPB = LEAN ? 1 : 2;
  static constexpr int BLOCKS_PER_SM = LEAN ? 11 : 1;
  // per warp: FP64 tiles, 1 / L_ii, then the lower triangle of a per-matrix
  // FP32 T_n (packed rows or tiles, in doubles rounded up to 16 bytes), which
  // doubles as the scratch tile of the L output (T_n is then not staged)
  static constexpr int off_rdiag = NTILE * 64;
  static constexpr int off_tstage = off_rdiag + DP;
  static constexpr int off_scratch = off_tstage;
  // T_n as packed rows, or as NTILE tiles of 64 floats (tiled inputs)
  static constexpr int tstage_rows = ((DP * (DP + 1) / 2 + 3) / 4) * 2;
  static constexpr int tstage = LEAN ? 0 : (tstage_rows > NTILE * 32 ? tstage_rows : NTILE * 32);
  static constexpr int off_mbar = off_tstage + tstage;  // one mbarrier (two doubles keep 16-byte alignment)
  static constexpr int per_warp = off_mbar + 2;
  static constexpr size_t smem = (size_t)WPB * per_warp * sizeof(double);
};

// A_ij + jt [i == j] in the model dtype (the rounding of the reference's
// separate tensor ops), as FP64; rows i >= D are the identity padding.
template <typename T>
__device__ __forceinline__ double assemble_one(T sv, T pv, bool has_p, T scale, T jt, int i, int c, int D) {
  if (i >= D) return (c == i) ? 1.0 : 0.0;
  if (c > i) return 0.0;
  T x = sv;
  if (has_p) x = add_rn(mul_rn(pv, scale), x);
  if (c == i) x = add_rn(x, jt);
  return (double)x;
}

// Lower tiles of A_n + jt I in FP64, padded with the identity, row block by
// row block with all loads of a block issued before any is used (coalesced:
// lanes read consecutive columns).  For FP32 with a per-matrix T_n, the lower
// triangle of T_n is copied to the packed FP32 stage in the same batches.
template <typename T, int DP>
__device__ __forceinline__ void assemble_tiles(const FactorArgs<T> &g, int64_t n, T scale, T jt, double *M,
                                               float *tstage, int lane) {
  constexpr int NT = DP / 8;
  constexpr int H = DP > 32 ? 2 : 1;
  const int D = g.D;
  const T *Sn = g.S + n * (int64_t)D * D;
  const T *Pn = g.P ? g.P + n * g.Pbs : nullptr;
  if constexpr (sizeof(T) == 4) {
    const float *Tn = tstage ? g.Tm + n * g.Tbs : nullptr;
#pragma unroll 1
    for (int I = 0; I < NT; ++I) {
      float sv[8][H], pv[8][H], tv[8][H];
#pragma unroll
      for (int rr = 0; rr < 8; ++rr) {
        const int i = 8 * I + rr;
#pragma unroll
        for (int h = 0; h < H; ++h) {
          const int c = lane + 32 * h;
          const bool in = i < D && c <= i;
          sv[rr][h] = in ? Sn[i * D + c] : 0.f;
          pv[rr][h] = (in && Pn) ? Pn[i * D + c] : 0.f;
          tv[rr][h] = (in && Tn) ? Tn[i * D + c] : 0.f;
        }
      }
#pragma unroll
      for (int rr = 0; rr < 8; ++rr) {
        const int i = 8 * I + rr;
#pragma unroll
        for (int h = 0; h < H; ++h) {
          const int c = lane + 32 * h;
          if (c >= 8 * I + 8) continue;  // right of the diagonal tile
          M[dmma::tix(I, c >> 3) + rr * 8 + (c & 7)] =
              assemble_one<T>(sv[rr][h], pv[rr][h], Pn != nullptr, scale, jt, i, c, D);
          if (Tn && i < D && c <= i) tstage[i * (i + 1) / 2 + c] = tv[rr][h];
        }
      }
    }
    __syncwarp();
  } else {
#pragma unroll 1
    for (int I = 0; I < NT; ++I) {
      T sv[8][H], pv[8][H];
#pragma unroll
      for (int rr = 0; rr < 8; ++rr) {
        const int i = 8 * I + rr;
#pragma unroll
        for (int h = 0; h < H; ++h) {
          const int c = lane + 32 * h;
          const bool in = i < D && c <= i;
          sv[rr][h] = in ? Sn[i * D + c] : T(0);
          pv[rr][h] = (in && Pn) ? Pn[i * D + c] : T(0);
        }
      }
#pragma unroll
      for (int rr = 0; rr < 8; ++rr) {
#pragma unroll
        for (int h = 0; h < H; ++h) {
          const int c = lane + 32 * h;
          if (c >= 8 * I + 8) continue;  // right of the diagonal tile
          M[dmma::tix(I, c >> 3) + rr * 8 + (c & 7)] =
              assemble_one<T>(sv[rr][h], pv[rr][h], Pn != nullptr, scale, jt, 8 * I + rr, c, D);
        }
      }
    }
    __syncwarp();
  }
}

// ---- tiled inputs: one bulk copy per matrix, converted in place ----------
__device__ __forceinline__ uint32_t sm_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

constexpr uint32_t kBulkSpinLimit = 1u << 26;

// Waits for the mbarrier phase; false once 1.5 s have passed (checked every
// 1024 polls) or after kBulkSpinLimit polls.
__device__ __forceinline__ bool bulk_wait(uint64_t *mbar, uint32_t parity) {
  const uint32_t a = sm_u32(mbar);
  uint64_t t0 = 0;
  for (uint32_t it = 0; it < kBulkSpinLimit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
    if ((it & 1023u) == 0) {
      uint64_t now;
      asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(now));
      if (it == 0) t0 = now;
      else if (now - t0 > 1500000000ull) return false;
    }
  }
  return false;
}

// Lane 0 issues the copies of SP_n (into the tile area) and T_n (into the T
// stage) on the warp's mbarrier; every lane first orders its earlier shared
// memory accesses before the asynchronous writes.
template <int DP, bool LEAN>
__device__ __forceinline__ void bulk_issue(const FactorArgs<float> &g, int64_t n, double *M, uint64_t *mbar, int lane) {
  using C = DmmaCfg<DP, LEAN>;
  constexpr uint32_t sp_bytes = C::NTILE * 512u, t_bytes = C::NTILE * 256u;
  const uint32_t total = sp_bytes + ((!LEAN && g.Tt) ? t_bytes : 0u);
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  __syncwarp();
  if (lane == 0) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(sm_u32(mbar)), "r"(total)
                 : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     sm_u32(M)),
                 "l"(g.SP + n * (int64_t)(C::NTILE * 128)), "r"(sp_bytes), "r"(sm_u32(mbar))
                 : "memory");
    if (!LEAN && g.Tt)
      asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                       sm_u32(M + C::off_tstage)),
                   "l"(g.Tt + n * (int64_t)(C::NTILE * 64)), "r"(t_bytes), "r"(sm_u32(mbar))
                   : "memory");
  }
}

// Row block of tile t = I (I + 1) / 2 + J of the lower tiles.
__host__ __device__ constexpr int tile_row(int t) {
  int I = 0;
  while ((I + 1) * (I + 2) / 2 <= t) ++I;
  return I;
}

// Tile t of the copied area holds S_t then P_t (128 floats = the 512 bytes
// of FP64 tile t).  Lane l takes the element pair 2 l, 2 l + 1 of every tile
// (row l / 4, columns 2 (l % 4) and + 1): a batch of NB tiles is read as
// float2 pairs, the warp synchronises, and the FP64 entries of A_n + jt I
// replace them as double2 pairs.  SP is zero outside D and above the
// diagonal, so only the diagonal tiles (jitter, identity padding) and the
// rows beyond D of the last row block need masks.
template <int DP>
__device__ __forceinline__ void convert_tiles(double *M, float scale, float jt, int D, int lane) {
  constexpr int NT = DP / 8, NTILE = NT * (NT + 1) / 2;
  constexpr int NB = 9;  // tiles per batch
  const float *F = reinterpret_cast<const float *>(M);
  const int r = lane >> 2, c = 2 * (lane & 3);
#pragma unroll
  for (int t0 = 0; t0 < NTILE; t0 += NB) {
    float2 sv[NB], pv[NB];
#pragma unroll
    for (int b = 0; b < NB; ++b) {
      if (t0 + b < NTILE) {
        sv[b] = *reinterpret_cast<const float2 *>(F + (t0 + b) * 128 + 2 * lane);
        pv[b] = *reinterpret_cast<const float2 *>(F + (t0 + b) * 128 + 64 + 2 * lane);
      }
    }
    __syncwarp();
#pragma unroll
    for (int b = 0; b < NB; ++b) {
      const int t = t0 + b;
      if (t < NTILE) {
        const int I = tile_row(t), J = t - I * (I + 1) / 2;
        const int i = 8 * I + r;
        const float x0 = add_rn(mul_rn(pv[b].x, scale), sv[b].x);
        const float x1 = add_rn(mul_rn(pv[b].y, scale), sv[b].y);
        double d0 = (double)x0, d1 = (double)x1;
        if (I == J) {
          const int j0 = 8 * J + c;
          d0 = (i >= D) ? (i == j0 ? 1.0 : 0.0) : (j0 > i ? 0.0 : (j0 == i ? (double)add_rn(x0, jt) : d0));
          d1 = (i >= D) ? (i == j0 + 1 ? 1.0 : 0.0)
                        : (j0 + 1 > i ? 0.0 : (j0 + 1 == i ? (double)add_rn(x1, jt) : d1));
        } else if (i >= D) {
          d0 = 0.0;
          d1 = 0.0;
        }
        *reinterpret_cast<double2 *>(M + t * 64 + 2 * lane) = make_double2(d0, d1);
      }
    }
    __syncwarp();
  }
}

// B fragments of the 8-column block Ac of T_n, tile K of rows 8K..8K+7:
// tb[K][s] = T[8K + 4s + t % 4][8 Ac + t / 4].
template <typename T, int NT>
__device__ __forceinline__ void load_tcol(const T *Tn, int D, int lower, int Ac, int lane, T (&tb)[NT][2]) {
  const int col = 8 * Ac + (lane >> 2);
#pragma unroll
  for (int K = 0; K < NT; ++K)
#pragma unroll
    for (int s = 0; s < 2; ++s) {
      const int row = 8 * K + 4 * s + (lane & 3);
      tb[K][s] = (row < D && col < D && (!lower || col <= row)) ? Tn[row * D + col] : T(0);
    }
}

template <typename T, int DP, bool LEAN>
__device__ __forceinline__ void factor_one(const FactorArgs<T> &g, int64_t n, double *M, int lane, uint32_t *phase,
                                           bool *halt) {
  using C = DmmaCfg<DP, LEAN>;
  constexpr int NT = C::NT;
  double *scratch = M + C::off_scratch;
  double *rdiag = M + C::off_rdiag;
  // per-matrix FP32 T_n goes through shared memory with the other inputs
  const bool tiled = sizeof(T) == 4 && g.SP != nullptr;
  const bool staged = !LEAN && sizeof(T) == 4 && !g.L && ((g.Tm && g.Tbs != 0) || (tiled && g.Tt));
  float *tstage = staged ? reinterpret_cast<float *>(M + C::off_tstage) : nullptr;
  const int D = g.D;
  const T scale = posterior_scale(g, n);
  T jit = g.jitter[n];
  T *lout = g.L ? g.L + n * (int64_t)D * D : nullptr;
  // tiled FP32 input with its T_n tiles staged: the trace runs inside the sweep
  const bool fused_trace = staged && tiled;
  double trace_acc = 0.0;
  bool ok = false;
  for (int attempt = 0; attempt <= 32 && !ok; ++attempt) {
    T jt = jit;
    if (attempt > 0) {
      jt = T(0);
      for (int k = 0; k < attempt; ++k) jt = add_rn(jt, (T)(g.eps * ldexp(1.0, k)));
    }
    if constexpr (sizeof(T) == 4) {
      if (tiled) {
        uint64_t *mbar = reinterpret_cast<uint64_t *>(M + C::off_mbar);
        bulk_issue<DP, LEAN>(g, n, M, mbar, lane);
        const bool arrived = bulk_wait(mbar, *phase);
        *phase ^= 1u;
        if (!arrived) {
          // no copy lands after a second bounded wait: the warp stops here
          bulk_wait(mbar, *phase ^ 1u);
          if (lane == 0) g.info[n] = -2;
          *halt = true;
          return;
        }
        convert_tiles<DP>(M, scale, jt, D, lane);
      } else {
        assemble_tiles<T, DP>(g, n, scale, jt, M, tstage, lane);
      }
    } else {
      assemble_tiles<T, DP>(g, n, scale, jt, M, tstage, lane);
    }
    __syncwarp();
    trace_acc = 0.0;
    ok = dmma::chol_inv_blocked<NT, T>(M, scratch, rdiag, lane, lout, D, fused_trace ? tstage : nullptr, trace_acc);
    if (ok) jit = jt;
    __syncwarp();
  }
  if (lane == 0) {
    g.jitter[n] = jit;
    g.info[n] = ok ? 0 : -1;
  }
  const T nanv = T(NAN);
  T *W = g.W ? g.W + n * (int64_t)D * D : nullptr;
  float *Xt = g.Xt ? g.Xt + n * (int64_t)(C::NTILE * 64) : nullptr;
  float *Wc = g.Wc ? g.Wc + n * (int64_t)(C::NTILE * 128) : nullptr;
  if (!ok) {
    for (int e = lane; e < D * D; e += 32) {
      if (W) W[e] = nanv;
      if (lout) lout[e] = nanv;
    }
    if (Xt)
      for (int e = lane; e < C::NTILE * 64; e += 32) Xt[e] = NAN;
    if (Wc)
      for (int e = lane; e < C::NTILE * 128; e += 32) Wc[e] = NAN;
    if (lane == 0) {
      g.logdet[n] = nanv;
      if (g.Tm || g.Tt) g.trace[n] = nanv;
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
  // first column block of a shared or FP64 T in flight during the W output
  const T *Tn = g.Tm ? g.Tm + n * g.Tbs : nullptr;
  T tb[NT][2];
  if (Tn && !staged) load_tcol<T, NT>(Tn, D, g.T_lower, 0, lane, tb);
  if (Xt) {
    // X as lower tiles, zero outside D (256 contiguous bytes per tile)
#pragma unroll 1
    for (int I = 0; I < NT; ++I)
#pragma unroll 1
      for (int J = 0; J <= I; ++J) {
        const int t = I * (I + 1) / 2 + J;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int e = lane + 32 * h;
          const int i = 8 * I + (e >> 3), j = 8 * J + (e & 7);
          Xt[t * 64 + e] = (i < D && j <= i) ? (float)M[t * 64 + e] : 0.f;
        }
      }
  }
  if (Wc) {
    // segment J holds the tf32 hi parts of the tiles I = J .. NT - 1 of
    // column block J, then their lo parts (tf32 of the rest), each tile as
    // two K-major cores (columns 8 J .. 8 J + 3, then 8 J + 4 .. 8 J + 7);
    // lane l writes row l / 4, column l % 4 of a core, so a warp store is one
    // contiguous 128-byte core.  Rows i >= D (the identity padding) are zero.
    const int rr = lane >> 2, cc = lane & 3;
#pragma unroll
    for (int J = 0; J < NT; ++J) {
      float *seg = Wc + 128 * (J * NT - J * (J - 1) / 2);
#pragma unroll
      for (int I = J; I < NT; ++I) {
        const int i = 8 * I + rr;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int j = 8 * J + 4 * h + cc;
          const double v = M[dmma::tix(I, J) + rr * 8 + 4 * h + cc];
          const float x = (i < D && j <= i) ? (float)v : 0.f;
          const float hi = tf32_rna(x);
          seg[(I - J) * 64 + h * 32 + lane] = hi;
          seg[(NT - J) * 64 + (I - J) * 64 + h * 32 + lane] = tf32_rna(x - hi);
        }
      }
    }
  }
  // W_triu = X^T: W tile (J, I) = X_IJ^T for I >= J, zero below; lanes write
  // 8 consecutive columns of 4 rows per store
  if (W) {
    const int r = lane & 7;
#pragma unroll 1
    for (int J = 0; J < NT; ++J) {
#pragma unroll
      for (int I = 0; I < NT; ++I) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int c = (lane >> 3) + 4 * h;
          const int row = 8 * J + c, col = 8 * I + r;
          if (row < D && col < D) {
            double v = 0.0;
            if (I > J || (I == J && r >= c)) v = M[dmma::tix(I, J) + r * 8 + c];
            W[row * D + col] = (T)v;
          }
        }
      }
    }
  }
  double ld = 0.0;
  for (int i = lane; i < D; i += 32) ld += log((double)(T)rdiag[i]);
  ld = warp_sum(ld);
  if (lane == 0) g.logdet[n] = (T)(2.0 * ld);
  if (fused_trace) {
    const double acc = warp_sum(trace_acc);
    if (lane == 0) g.trace[n] = (T)acc;
  } else if (staged) {
    // ||X T_n||_F^2 with X lower: (X T)_IA = sum_{K <= I} X_IK T_KA, column
    // block by column block; lower tiles of T_n (K >= A) from shared memory,
    // upper ones from global memory unless T_n is declared lower triangular
    const float *st = tstage;
    double acc = 0.0;
#pragma unroll 1
    for (int Ac = 0; Ac < NT; ++Ac) {
      const int col = 8 * Ac + (lane >> 2);
      double cacc[NT][2];
#pragma unroll
      for (int I = 0; I < NT; ++I) {
        cacc[I][0] = 0.0;
        cacc[I][1] = 0.0;
      }
#pragma unroll
      for (int K = 0; K < NT; ++K) {
        double b0 = 0.0, b1 = 0.0;
        const int r0 = 8 * K + (lane & 3), r1 = r0 + 4;
        if (K >= Ac && tiled) {
          // tile (K, Ac): local row lane % 4 (+ 4), local column lane / 4
          const float *tk = st + (K * (K + 1) / 2 + Ac) * 64 + (lane & 3) * 8 + (lane >> 2);
          b0 = (double)tk[0];
          b1 = (double)tk[32];
        } else if (K >= Ac) {
          b0 = (r0 < D && col <= r0) ? (double)st[r0 * (r0 + 1) / 2 + col] : 0.0;
          b1 = (r1 < D && col <= r1) ? (double)st[r1 * (r1 + 1) / 2 + col] : 0.0;
        } else {
          if (g.T_lower || tiled) continue;
          b0 = (r0 < D && col < D) ? (double)Tn[r0 * D + col] : 0.0;
          b1 = (r1 < D && col < D) ? (double)Tn[r1 * D + col] : 0.0;
          if (!__any_sync(0xffffffffu, b0 != 0.0 || b1 != 0.0)) continue;
        }
#pragma unroll
        for (int I = K; I < NT; ++I) {
          const double *x = M + dmma::tix(I, K);
          dmma::mma(cacc[I][0], cacc[I][1], dmma::afrag(x, 0, lane), b0);
          dmma::mma(cacc[I][0], cacc[I][1], dmma::afrag(x, 1, lane), b1);
        }
      }
#pragma unroll
      for (int I = 0; I < NT; ++I) acc = fma(cacc[I][0], cacc[I][0], fma(cacc[I][1], cacc[I][1], acc));
    }
    acc = warp_sum(acc);
    if (lane == 0) g.trace[n] = (T)acc;
  } else if (tiled && g.Tt) {
    // the same product with the tiles of T_n read from global memory (the
    // lean form stages none): column block Ac + 1's B fragments are loaded
    // while block Ac's products run
    const float *tt = reinterpret_cast<const float *>(g.Tt) + n * (int64_t)(C::NTILE * 64);
    const int fo = (lane & 3) * 8 + (lane >> 2);
    float tb[NT][2];
#pragma unroll
    for (int K = 0; K < NT; ++K) {
      tb[K][0] = tt[(K * (K + 1) / 2) * 64 + fo];
      tb[K][1] = tt[(K * (K + 1) / 2) * 64 + fo + 32];
    }
    double acc = 0.0;
#pragma unroll 1
    for (int Ac = 0; Ac < NT; ++Ac) {
      double b[NT][2];
#pragma unroll
      for (int K = 0; K < NT; ++K) {
        b[K][0] = (double)tb[K][0];
        b[K][1] = (double)tb[K][1];
      }
      if (Ac + 1 < NT) {
#pragma unroll
        for (int K = 0; K < NT; ++K) {
          if (K >= Ac + 1) {
            tb[K][0] = tt[(K * (K + 1) / 2 + Ac + 1) * 64 + fo];
            tb[K][1] = tt[(K * (K + 1) / 2 + Ac + 1) * 64 + fo + 32];
          }
        }
      }
      double cacc[NT][2];
#pragma unroll
      for (int I = 0; I < NT; ++I) {
        cacc[I][0] = 0.0;
        cacc[I][1] = 0.0;
      }
#pragma unroll
      for (int K = 0; K < NT; ++K) {
        if (K < Ac) continue;
#pragma unroll
        for (int I = K; I < NT; ++I) {
          const double *x = M + dmma::tix(I, K);
          dmma::mma(cacc[I][0], cacc[I][1], dmma::afrag(x, 0, lane), b[K][0]);
          dmma::mma(cacc[I][0], cacc[I][1], dmma::afrag(x, 1, lane), b[K][1]);
        }
      }
#pragma unroll
      for (int I = 0; I < NT; ++I) acc = fma(cacc[I][0], cacc[I][0], fma(cacc[I][1], cacc[I][1], acc));
    }
    acc = warp_sum(acc);
    if (lane == 0) g.trace[n] = (T)acc;
  } else if (Tn) {
    // ||X T_n||_F^2 with X lower: (X T)_IA = sum_{K <= I} X_IK T_KA, column
    // block by column block, the next block's loads issued before this one's
    // products; all-zero tiles of T_n (its upper part when triangular) skipped
    double acc = 0.0;
#pragma unroll 1
    for (int Ac = 0; Ac < NT; ++Ac) {
      double b[NT][2];
      unsigned nonzero = 0;
#pragma unroll
      for (int K = 0; K < NT; ++K) {
        b[K][0] = (double)tb[K][0];
        b[K][1] = (double)tb[K][1];
        if (__any_sync(0xffffffffu, b[K][0] != 0.0 || b[K][1] != 0.0)) nonzero |= 1u << K;
      }
      if (Ac + 1 < NT) load_tcol<T, NT>(Tn, D, g.T_lower, Ac + 1, lane, tb);
#pragma unroll
      for (int I = 0; I < NT; ++I) {
        double c0 = 0.0, c1 = 0.0;
        asm volatile("" ::: "memory");
#pragma unroll
        for (int K = 0; K <= I; ++K) {
          if (!((nonzero >> K) & 1u)) continue;
          const double *x = M + dmma::tix(I, K);
          dmma::mma(c0, c1, dmma::afrag(x, 0, lane), b[K][0]);
          dmma::mma(c0, c1, dmma::afrag(x, 1, lane), b[K][1]);
        }
        acc = fma(c0, c0, fma(c1, c1, acc));
      }
    }
    acc = warp_sum(acc);
    if (lane == 0) g.trace[n] = (T)acc;
  }
}

// Persistent: each warp walks matrices n, n + stride, ... (a grid of exactly
// the resident blocks).
template <typename T, int DP, bool LEAN>
__global__ void __launch_bounds__(32 * DmmaCfg<DP, LEAN>::WPB, DmmaCfg<DP, LEAN>::BLOCKS_PER_SM)
    factor_dmma_kernel(FactorArgs<T> g) {
  using C = DmmaCfg<DP, LEAN>;
  extern __shared__ double smem_d[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double *M = smem_d + warp * C::per_warp;
  const int64_t stride = (int64_t)gridDim.x * C::WPB;
  uint32_t phase = 0;
  bool halt = false;
  if (lane == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"((uint32_t)__cvta_generic_to_shared(M + C::off_mbar))
                 : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncwarp();
  for (int64_t n = (int64_t)blockIdx.x * C::WPB + warp; n < g.N && !halt; n += stride) {
    factor_one<T, DP, LEAN>(g, n, M, lane, &phase, &halt);
    __syncwarp();
  }
}

}  // namespace lakde

using namespace lakde;

// Persistent DMMA launch: exactly the blocks that are resident at once
// (registers and shared memory), so every block starts immediately.
template <typename TT, int DP, bool LEAN>
static int launch_factor_dmma_v(const FactorArgs<TT> &g, int64_t N, void *stream) {
  using C = DmmaCfg<DP, LEAN>;
  auto kern = factor_dmma_kernel<TT, DP, LEAN>;
  if (C::smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::smem);
    if (e != cudaSuccess) {
      set_error("posterior_factor: %s", cudaGetErrorString(e));
      return (int)LAKDE_ECUDA;
    }
  }
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1) sms = 148;
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 32 * C::WPB, C::smem) != cudaSuccess ||
      per_sm < 1) {
    cudaGetLastError();
    per_sm = 1;
  }
  int64_t blocks = (N + C::WPB - 1) / C::WPB;
  if (blocks > (int64_t)sms * per_sm) blocks = (int64_t)sms * per_sm;
  kern<<<(unsigned)blocks, 32 * C::WPB, C::smem, as_stream(stream)>>>(g);
  return check_launch("posterior_factor");
}

// The lean variant (no staged T_n: tiles of T_n are read from global memory)
// when the call writes no L, takes no dense T_n, and the tuning table selects
// it (lakde_tuning_set, knob LAKDE_TUNE_FACTOR).
template <typename TT, int DP>
static int launch_factor_dmma(const FactorArgs<TT> &g, int64_t N, void *stream) {
  const bool lean_ok = !g.L && !g.Tm;
  if (lean_ok && tuning(LAKDE_TUNE_FACTOR, g.D) == 1) return launch_factor_dmma_v<TT, DP, true>(g, N, stream);
  return launch_factor_dmma_v<TT, DP, false>(g, N, stream);
}

extern "C" int lakde_posterior_factor(int dtype, int64_t N, int64_t D, const void *S, const void *P,
                                      int64_t P_batch_stride, const void *nu_0, const void *a, const void *b,
                                      void *jitter, double eps, void *W_triu, void *L, void *logdet_W,
                                      int32_t *info, const void *T, int64_t T_batch_stride, int T_lower,
                                      void *trace, void *W_cores, void *stream) {
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
  if (W_cores && (dtype != LAKDE_F32 || (reinterpret_cast<uintptr_t>(W_cores) & 15u))) {
    set_error("posterior_factor: W_cores needs float32 values and a 16-byte aligned buffer");
    return LAKDE_EINVAL;
  }
  if (int st = bind_device("posterior_factor",
                           {W_triu, S, P, nu_0, a, b, jitter, L, logdet_W, info, T, trace, W_cores}))
    return st;
  return dispatch_float(dtype, [&](auto t0) {
    using TT = decltype(t0);
    FactorArgs<TT> g{};
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
    g.T_lower = T_lower != 0;
    g.trace = static_cast<TT *>(trace);
    if constexpr (sizeof(TT) == 4) g.Wc = static_cast<float *>(W_cores);
    g.N = N;
    g.D = (int)D;
    return dispatch_dp(D, [&](auto dp) {
      constexpr int DP = decltype(dp)::value;
      if constexpr (DP <= 8) {
        factor_thread_kernel<TT, DP><<<(unsigned)((N + 127) / 128), 128, 0, as_stream(stream)>>>(g);
        if (int st = check_launch("posterior_factor")) return st;
        // the register kernel writes W_triu only: its cores by the packing kernel
        if (W_cores) return lakde_pack_w_cores(LAKDE_F32, N, D, W_triu, W_cores, stream);
        return (int)LAKDE_OK;
      } else {
        return launch_factor_dmma<TT, DP>(g, N, stream);
      }
    });
  });
}

// ------------------------------------------------------------- tiled layout
extern "C" int64_t lakde_tile_count(int64_t D) {
  int64_t nt = 0;
  if (D >= 1 && D <= kMaxDim) {
    dispatch_dp(D, [&](auto dp) {
      nt = decltype(dp)::value / 8;
      return 0;
    });
  }
  return nt * (nt + 1) / 2;
}

template <typename T>
__global__ void pack_tiles_kernel(const T *__restrict__ src, int64_t sbs, T *__restrict__ dst, int64_t dbs,
                                  int64_t dts, int64_t doff, int64_t N, int D, int NT) {
  const int ntile = NT * (NT + 1) / 2;
  const int64_t total = N * ntile * 64;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < total; k += (int64_t)gridDim.x * blockDim.x) {
    const int e = (int)(k & 63);
    const int64_t rest = k >> 6;
    const int t = (int)(rest % ntile);
    const int64_t n = rest / ntile;
    int I = 0;
    while ((I + 1) * (I + 2) / 2 <= t) ++I;
    const int J = t - I * (I + 1) / 2;
    const int i = 8 * I + (e >> 3), j = 8 * J + (e & 7);
    const T v = (i < D && j < D && j <= i) ? src[n * sbs + (int64_t)i * D + j] : T(0);
    dst[n * dbs + (int64_t)t * dts + doff + e] = v;
  }
}

extern "C" int lakde_pack_tiles(int dtype, int64_t N, int64_t D, const void *src, int64_t src_batch_stride,
                                void *dst, int64_t dst_batch_stride, int64_t dst_tile_stride, int64_t dst_offset,
                                void *stream) {
  clear_error();
  if (N < 0 || D < 1 || D > kMaxDim || dst_tile_stride < 64 || dst_offset < 0) {
    set_error("pack_tiles: invalid sizes");
    return LAKDE_EINVAL;
  }
  if (N == 0) return LAKDE_OK;
  if (!src || !dst) {
    set_error("pack_tiles: null pointer");
    return LAKDE_EINVAL;
  }
  if (int st = bind_device("pack_tiles", {dst, src})) return st;
  const int64_t ntile = lakde_tile_count(D);
  int NT = 0;
  while (NT * (NT + 1) / 2 < ntile) ++NT;
  return dispatch_float(dtype, [&](auto t0) {
    using T = decltype(t0);
    const int64_t total = N * ntile * 64;
    int64_t blocks = (total + 255) / 256;
    if (blocks > 148 * 32) blocks = 148 * 32;
    pack_tiles_kernel<T><<<(unsigned)blocks, 256, 0, as_stream(stream)>>>(
        static_cast<const T *>(src), src_batch_stride, static_cast<T *>(dst), dst_batch_stride, dst_tile_stride,
        dst_offset, N, (int)D, NT);
    return check_launch("pack_tiles");
  });
}

extern "C" int lakde_posterior_factor_tiled(int dtype, int64_t N, int64_t D, const void *SP, const void *nu_0,
                                            const void *a, const void *b, void *jitter, double eps, void *W_triu,
                                            void *X_tiles, void *W_cores, void *logdet_W, int32_t *info,
                                            const void *T_tiles, void *trace, void *stream) {
  clear_error();
  if (dtype != LAKDE_F32) {
    set_error("posterior_factor_tiled: float32 values only");
    return LAKDE_EDTYPE;
  }
  if (N < 0 || D <= 8 || D > kMaxDim) {
    set_error("posterior_factor_tiled: needs 8 < D <= %d (N=%lld, D=%lld)", kMaxDim, (long long)N, (long long)D);
    return LAKDE_EUNSUPPORTED;
  }
  if (N == 0) return LAKDE_OK;
  if (!SP || !nu_0 || !a || !b || !jitter || (!W_triu && !X_tiles && !W_cores) || !logdet_W || !info ||
      (T_tiles && !trace)) {
    set_error("posterior_factor_tiled: missing buffer");
    return LAKDE_EINVAL;
  }
  if (N > 0x7fffffffLL) {
    set_error("posterior_factor_tiled: N too large");
    return LAKDE_EUNSUPPORTED;
  }
  if ((reinterpret_cast<uintptr_t>(SP) | reinterpret_cast<uintptr_t>(T_tiles) | reinterpret_cast<uintptr_t>(W_cores)) &
      15u) {
    set_error("posterior_factor_tiled: SP, T_tiles and W_cores must be 16-byte aligned");
    return LAKDE_EINVAL;
  }
  if (int st = bind_device("posterior_factor_tiled",
                           {SP, W_triu, X_tiles, W_cores, nu_0, a, b, jitter, logdet_W, info, T_tiles, trace}))
    return st;
  FactorArgs<float> g{};
  g.SP = static_cast<const float *>(SP);
  g.Tt = static_cast<const float *>(T_tiles);
  g.nu0 = static_cast<const float *>(nu_0);
  g.a = static_cast<const float *>(a);
  g.b = static_cast<const float *>(b);
  g.jitter = static_cast<float *>(jitter);
  g.eps = eps;
  g.W = static_cast<float *>(W_triu);
  g.Xt = static_cast<float *>(X_tiles);
  g.Wc = static_cast<float *>(W_cores);
  g.logdet = static_cast<float *>(logdet_W);
  g.info = info;
  g.T_lower = 1;
  g.trace = static_cast<float *>(trace);
  g.N = N;
  g.D = (int)D;
  return dispatch_dp(D, [&](auto dp) {
    constexpr int DP = decltype(dp)::value;
    if constexpr (DP <= 8) {
      return (int)LAKDE_EUNSUPPORTED;
    } else {
      return launch_factor_dmma<float, DP>(g, N, stream);
    }
  });
}
