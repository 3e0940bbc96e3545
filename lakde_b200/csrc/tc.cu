// Mixed-precision tensor-core (tcgen05) kernels of the large-D VI path.
//
// Grouping pairs by kernel makes two dense contractions per kernel row n with
// m_n pairs, Delta = [x_m - x_n] (m_n x D):
//   E-step  Y = Delta W_triu_n          (m_n x D), Q_p = |Y_p|^2   (lakde/local_adaptive_kde.py:36-44)
//   M-step  S_n = G^T G, G = sqrt(r) Delta                          (lakde/local_adaptive_kde.py:66-81)
// Both run as tcgen05.mma kind::f16 on bf16 operands with fp32 accumulation in
// tensor memory.  A split x = hi + lo (hi = bf16(x), lo = bf16(x - hi)) keeps
// ~16 significant bits: each product is hi*hi + lo*hi + hi*lo.  The
// differences are centred on the kernel in fp32 before the split, so the
// cancellation near each kernel centre happens in fp32, not in bf16.
//
// Operands are staged by the CTA's threads into shared memory in the canonical
// no-swizzle core-matrix layout (8 rows x 16 bytes per core matrix).  One
// thread issues the MMAs; completion is signalled through an mbarrier whose
// waits are bounded (on timeout the kernel raises an error flag and stops).
// D is padded to 64 (zero rows and columns).
#include <cuda_bf16.h>

#include "common.cuh"

namespace lakde {
namespace tc {

constexpr int DP = 64;       // padded dimension
constexpr int KG = DP / 8;   // 8-element groups along D
constexpr int MT = 128;      // pairs per tile (MMA M for the E-step)
constexpr uint32_t kSpinLimit = 1u << 24;

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor: no swizzle, version 1 (sm_100).
__device__ __forceinline__ uint64_t desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | ((uint64_t)1 << 46);
}

// Instruction descriptor, kind::f16: bf16 x bf16 -> f32, M x N, operand majors.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N, int a_mn_major, int b_mn_major) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)a_mn_major << 15) | ((uint32_t)b_mn_major << 16) |
         ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void commit(uint64_t *mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(mbar))
               : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t *mbar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(mbar)) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ bool mbar_wait(uint64_t *mbar, uint32_t parity) {
  const uint32_t addr = smem_u32(mbar);
  for (uint32_t it = 0; it < kSpinLimit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(addr), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)), "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// 16 consecutive fp32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// hi = bf16(x), lo = bf16(x - hi), packed pairwise (x0 in the low half); the
// pair conversions are one instruction each
__device__ __forceinline__ void split2(float x0, float x1, uint32_t &hi, uint32_t &lo) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(x0, x1);
  const float2 hf = __bfloat1622float2(h);
  const __nv_bfloat162 l = __floats2bfloat162_rn(x0 - hf.x, x1 - hf.y);
  hi = *reinterpret_cast<const uint32_t *>(&h);
  lo = *reinterpret_cast<const uint32_t *>(&l);
}

// byte offset of element (row, d) of a [rows x DP] bf16 operand in core-matrix
// layout with the 8-row groups `rstride` bytes apart and the 8-column groups
// 128 bytes apart:  core (row / 8, d / 8) + 16 (row % 8) + 2 (d % 8)
__device__ __forceinline__ uint32_t core_off(int row, int d, uint32_t rstride) {
  return (uint32_t)(row >> 3) * rstride + (uint32_t)(d >> 3) * 128u + (uint32_t)(row & 7) * 16u + (uint32_t)(d & 7) * 2u;
}

struct TcArgs {
  const int64_t *rowptr;
  const int32_t *col;
  const int32_t *order;
  const float *r;
  const float *X;
  const float *W;       // W_triu [N, D, D]
  const float *nu;      // E-step: per-kernel nu
  const float *logdet;  // E-step
  float *logrho;        // E-step output
  float *S;             // M-step output [N, D, D]
  float *nu_out;        // M-step output
  int lower_only;       // M-step: write only j <= i of S_n
  float *SPo;           // M-step: S_n as lower 8 x 8 tiles into the S halves of SP
  const uint32_t *Wc;   // E-step: W_triu_n as bf16 hi / lo B-operand core segments (instead of W)
  int nt;               // E-step with Wc: 8-row tile blocks of the tiled layout
  int ntile;
  float nu0;
  int64_t npts;
  int64_t N;
  int64_t koff;  // row n is kernel n + koff of X
  int D;
  int *err;
};

// --------------------------------------------------------------------- E-step
// smem: A_hi, A_lo [MT x DP] (K-major: pair rows), B_hi, B_lo [DP x DP] (MN-major:
// rows of W_triu), cidx[MT], mbarrier, tmem slot.
struct EsmCfg {
  static constexpr uint32_t A_BYTES = MT * DP * 2;   // 16 KB
  static constexpr uint32_t B_BYTES = DP * DP * 2;   // 8 KB
  static constexpr uint32_t off_Ahi = 0, off_Alo = A_BYTES, off_Bhi = 2 * A_BYTES, off_Blo = 2 * A_BYTES + B_BYTES;
  static constexpr uint32_t off_c = 2 * A_BYTES + 2 * B_BYTES;
  static constexpr uint32_t bytes = off_c + MT * 4 + 128;
};

// Bulk copy of W_triu_n's B cores (WC layout) into B_hi / B_lo: segment J
// (cores I = J .. nt - 1, hi then lo) lands at core (J, J) of each, i.e.
// J * (KG + 1) * 128 bytes in.  One thread issues; the cores above the block
// diagonal and outside nt stay zero from the kernel's start.
__device__ __forceinline__ void issue_b_cores(const uint32_t *src, int nt, uint32_t bhi, uint32_t blo,
                                              uint64_t *bar) {
  const uint32_t total = (uint32_t)(nt * (nt + 1) / 2) * 256u;
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(total) : "memory");
  const unsigned char *p = reinterpret_cast<const unsigned char *>(src);
  for (int J = 0; J < nt; ++J) {
    const uint32_t bytes = (uint32_t)(nt - J) * 128u, o = (uint32_t)J * (KG + 1) * 128u;
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     bhi + o),
                 "l"(p), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     blo + o),
                 "l"(p + bytes), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
    p += 2 * bytes;
  }
}

template <bool WC>
__global__ void __launch_bounds__(128, 4) estep_tc_kernel(TcArgs g) {
  using C = EsmCfg;
  extern __shared__ __align__(128) unsigned char sm[];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ __align__(8) uint64_t bbar;
  __shared__ uint32_t s_tmem;
  __shared__ float s_cst, s_expo;
  unsigned char *Ahi = sm + C::off_Ahi, *Alo = sm + C::off_Alo, *Bhi = sm + C::off_Bhi, *Blo = sm + C::off_Blo;
  int32_t *cidx = reinterpret_cast<int32_t *>(sm + C::off_c);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int D = g.D;

  if (warp == 0) tmem_alloc(&s_tmem, 64);
  if (tid == 0) {
    mbar_init(&mbar);
    if (WC) {
      mbar_init(&bbar);
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
  }
  if (WC) {
    // B cores that no copy writes (above the block diagonal, outside nt) are
    // zero; the copied ones are left to the copies
    uint4 *bz = reinterpret_cast<uint4 *>(Bhi);
    for (int e = tid; e < (int)(2 * C::B_BYTES / 16); e += 128) {
      const int core = (e >> 3) & (KG * KG - 1), J = core / KG, I = core % KG;
      if (I < J || I >= g.nt || J >= g.nt) bz[e] = make_uint4(0u, 0u, 0u, 0u);
    }
    fence_async_smem();
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = s_tmem;
  uint32_t phase = 0, bphase = 0;
  bool alive = true;

  // A: K-major, pair groups 8 * 128 bytes apart (SBO), K groups 128 bytes apart (LBO)
  // B: MN-major, N groups 128 bytes apart (SBO), K groups 8 * 128 bytes apart (LBO)
  constexpr uint32_t A_SBO = KG * 128, A_LBO = 128;
  constexpr uint32_t B_SBO = 128, B_LBO = KG * 128;
  const uint32_t idesc = idesc_bf16(MT, DP, 0, 1);
  // this thread's dimensions: 8 k + 2 (lane % 4) and + 1, k = 0 .. KG - 1
  const int dq = 2 * (lane & 3);

  // the next row's index and CSR bounds are loaded one row ahead
  int64_t it = blockIdx.x;
  int64_t n_nx = 0, start_nx = 0, end_nx = 0;
  if (it < g.N) {
    n_nx = g.order ? (int64_t)g.order[it] : it;
    start_nx = g.rowptr[n_nx];
    end_nx = g.rowptr[n_nx + 1];
  }
  for (; it < g.N && alive; it += gridDim.x) {
    const int64_t n = n_nx, start = start_nx, end = end_nx;
    const int64_t it2 = it + gridDim.x;
    if (it2 < g.N) {
      n_nx = g.order ? (int64_t)g.order[it2] : it2;
      start_nx = g.rowptr[n_nx];
      end_nx = g.rowptr[n_nx + 1];
    }
    // loads of the row, all issued before use: W_triu[n] (staged below as
    // B = [K = j][N = i], hi and lo), this thread's coordinates of x_n, and
    // nu_n / logdet_n for warp 0
    float wv[DP * DP / 256][2];
    if (WC) {
      // W_triu_n's cores by bulk copy: the previous row's MMAs have completed
      // (their mbarrier wait) and every thread has passed the row-end barrier
      if (tid == 0 && end > start) {
        fence_async_smem();
        issue_b_cores(g.Wc + n * (int64_t)(g.ntile * 64), g.nt, smem_u32(Bhi), smem_u32(Blo), &bbar);
      }
    } else {
      const float *Wn = g.W + n * (int64_t)D * D;
#pragma unroll
      for (int m = 0; m < DP * DP / 256; ++m) {
        const int e = tid + 128 * m;
        const int q = e >> 5, ln = e & 31;  // q: (jg, ig) block of 8 x 8
        const int j = 8 * (q / KG) + (ln >> 2), i = 8 * (q % KG) + 2 * (ln & 3);
        wv[m][0] = (j < D && i < D) ? Wn[j * D + i] : 0.f;
        wv[m][1] = (j < D && i + 1 < D) ? Wn[j * D + i + 1] : 0.f;
      }
    }
    const float *xnp = g.X + (n + g.koff) * (int64_t)D;
    float xn[KG][2];
#pragma unroll
    for (int k = 0; k < KG; ++k) {
      const int d0 = 8 * k + dq;
      xn[k][0] = d0 < D ? xnp[d0] : 0.f;
      xn[k][1] = d0 + 1 < D ? xnp[d0 + 1] : 0.f;
    }
    float nv = 0.f, ldn = 0.f;
    if (warp == 0) {
      nv = g.nu[n];
      ldn = g.logdet[n];
    }
    // B is written once per row: the previous row's last MMAs have completed
    // (their mbarrier wait) and every thread has passed the row-end barrier
    if (!WC && end > start) {
#pragma unroll
      for (int m = 0; m < DP * DP / 256; ++m) {
        const int e = tid + 128 * m;
        const int q = e >> 5, ln = e & 31;
        const int j = 8 * (q / KG) + (ln >> 2), i = 8 * (q % KG) + 2 * (ln & 3);
        uint32_t hi, lo;
        split2(wv[m][0], wv[m][1], hi, lo);
        // B is MN-major: core (k group j/8, n group i/8), 16-byte line = row j of 8 n's
        const uint32_t o = (uint32_t)(j >> 3) * B_LBO + (uint32_t)(i >> 3) * B_SBO + (uint32_t)(j & 7) * 16u +
                           (uint32_t)(i & 7) * 2u;
        *reinterpret_cast<uint32_t *>(Bhi + o) = hi;
        *reinterpret_cast<uint32_t *>(Blo + o) = lo;
      }
    }
    bool first = true;
    for (int64_t base = start; base < end; base += MT) {
      const int cnt = (int)((end - base) < MT ? (end - base) : MT);
      // gather: warp w takes the 8-row batches w, w + 4, w + 8, w + 12; lane
      // l the row 8 b + l / 4 and, for each 8-dimension group k, dimensions
      // 8 k + 2 (l % 4) and + 1.  Every store instruction then covers 8 rows
      // of one core-matrix column (32 distinct banks).  All column indices,
      // then all coordinates, are loaded before any is used.
      constexpr int NB = MT / 32;
      int32_t cb[NB];
#pragma unroll
      for (int b = 0; b < NB; ++b) {
        const int p = 8 * (warp + 4 * b) + (lane >> 2);
        int32_t c = -1;
        if (p < cnt) {
          c = g.col[base + p];
          if (c < 0 || c >= g.npts) c = -1;
        }
        cb[b] = c;
      }
      float v[NB][KG][2];
#pragma unroll
      for (int b = 0; b < NB; ++b) {
        const float *xm = g.X + (int64_t)(cb[b] < 0 ? 0 : cb[b]) * D;
#pragma unroll
        for (int k = 0; k < KG; ++k) {
          const int d0 = 8 * k + dq;
          v[b][k][0] = (cb[b] >= 0 && d0 < D) ? xm[d0] : 0.f;
          v[b][k][1] = (cb[b] >= 0 && d0 + 1 < D) ? xm[d0 + 1] : 0.f;
        }
      }
      if (first) {
        if (warp == 0) {
          // multivariate digamma, one term per lane
          double md = 0.0;
          for (int i = 1 + lane; i <= D; i += 32) md += digamma_d(0.5 * (double)nv + 0.5 * (1 - i));
          md = warp_sum(md);
          if (lane == 0) {
            s_cst = (float)(0.5 * (md + D * 0.69314718055994530942 + (double)ldn));
            s_expo = -0.5f * nv;
          }
        }
        first = false;
      }
#pragma unroll
      for (int b = 0; b < NB; ++b) {
        const int p = 8 * (warp + 4 * b) + (lane >> 2);
        if ((lane & 3) == 0) cidx[p] = cb[b];
#pragma unroll
        for (int k = 0; k < KG; ++k) {
          const int d0 = 8 * k + dq;
          const float x0 = cb[b] >= 0 ? v[b][k][0] - xn[k][0] : 0.f;
          const float x1 = cb[b] >= 0 ? v[b][k][1] - xn[k][1] : 0.f;
          uint32_t hi, lo;
          split2(x0, x1, hi, lo);
          const uint32_t o = core_off(p, d0, A_SBO);
          *reinterpret_cast<uint32_t *>(Ahi + o) = hi;
          *reinterpret_cast<uint32_t *>(Alo + o) = lo;
        }
      }
      fence_async_smem();
      fence_before();
      if (WC && base == start) {
        // the row's B cores have landed (every thread observes the mbarrier)
        const bool bok = __syncthreads_and(mbar_wait(&bbar, bphase) ? 1 : 0) != 0;
        bphase ^= 1;
        if (!bok) {
          // a copy still in flight may land later: wait once more before leaving
          mbar_wait(&bbar, bphase ^ 1);
          if (tid == 0) atomicExch(g.err, 1);
          alive = false;
          break;
        }
      } else {
        __syncthreads();
      }
      if (tid == 0) {
        fence_after();
        const uint32_t ahi = smem_u32(Ahi), alo = smem_u32(Alo), bhi = smem_u32(Bhi), blo = smem_u32(Blo);
#pragma unroll
        for (int s = 0; s < DP / 16; ++s) {
          const uint32_t ao = 2 * s * A_LBO, bo = 2 * s * B_LBO;
          mma(tmem, desc(ahi + ao, A_LBO, A_SBO), desc(bhi + bo, B_LBO, B_SBO), idesc, s > 0);
          mma(tmem, desc(alo + ao, A_LBO, A_SBO), desc(bhi + bo, B_LBO, B_SBO), idesc, 1);
          mma(tmem, desc(ahi + ao, A_LBO, A_SBO), desc(blo + bo, B_LBO, B_SBO), idesc, 1);
        }
        commit(&mbar);
      }
      // the outcome is made uniform across the CTA: the TMEM loads below are
      // warp-collective
      const bool ok = __syncthreads_and(mbar_wait(&mbar, phase) ? 1 : 0) != 0;
      phase ^= 1;
      fence_after();
      if (!ok) {
        if (tid == 0) atomicExch(g.err, 1);
        alive = false;
      }
      // epilogue: lane = pair row
      float q = 0.f;
      if (ok) {
        const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll
        for (int c0 = 0; c0 < DP; c0 += 16) {
          float vv[16];
          tmem_ld16(taddr + c0, vv);
#pragma unroll
          for (int k = 0; k < 16; ++k) q = fmaf(vv[k], vv[k], q);
        }
      }
      if (tid < cnt) {
        const int32_t c = cidx[tid];
        float lr = NAN;
        if (ok && c >= 0) {
          lr = __fadd_rn(__fmul_rn(q, s_expo), s_cst);
          if ((int64_t)c == n + g.koff) lr = -INFINITY;
        }
        g.logrho[base + tid] = lr;
      }
      fence_before();
      __syncthreads();
      if (!ok) break;
    }
    __syncthreads();
  }
  __syncthreads();
  fence_after();
  if (warp == 0) tmem_dealloc(tmem, 64);
}

// --------------------------------------------------------------------- M-step
// smem: G = [MT pairs x (hi | lo) 2 DP] bf16 (core rows of 16 groups); after
// the MMAs the accumulator rows [128 x RSTR] fp32 reuse it.
struct MsmCfg {
  static constexpr uint32_t G_BYTES = MT * 2 * DP * 2;  // 32 KB
  // row stride of the accumulator copy: 68 floats keeps the 16-byte row
  // writes of 8 consecutive threads on distinct bank groups
  static constexpr int RSTR = DP + 4;
  static constexpr uint32_t RED_BYTES = 128 * RSTR * 4;  // 34 KB
  static constexpr uint32_t bytes = (G_BYTES > RED_BYTES ? G_BYTES : RED_BYTES) + 128;
};

__global__ void __launch_bounds__(128, 4) mstep_tc_kernel(TcArgs g) {
  using C = MsmCfg;
  extern __shared__ __align__(128) unsigned char sm[];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t s_tmem;
  __shared__ float s_rs[4];
  unsigned char *G = sm;
  float *red = reinterpret_cast<float *>(sm);  // [128][RSTR] after the MMAs
  constexpr int RSTR = C::RSTR;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int D = g.D;

  if (warp == 0) tmem_alloc(&s_tmem, 64);
  if (tid == 0) mbar_init(&mbar);
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = s_tmem;
  uint32_t phase = 0;
  bool alive = true;

  // G rows are pairs: core (pair group, dim group 0..15), dim groups 0-7 hi, 8-15 lo.
  // As A = [G_hi^T; G_lo^T] (M = 128 dims, K = pairs) and B = G_hi (K = pairs,
  // N = 64 dims) both are MN-major: MN groups 128 bytes apart (SBO), K (pair)
  // groups 16 * 128 bytes apart (LBO).  The accumulator holds H = G_hi^T G_hi
  // (rows 0-63) and B = G_lo^T G_hi (rows 64-127); G_hi^T G_lo = B^T, so
  // S = H + B + B^T (the lo * lo term is below the split's precision).
  constexpr uint32_t RS = 2 * KG * 128;  // pair-group stride
  constexpr uint32_t SBO = 128, LBO = RS;
  const uint32_t idesc = idesc_bf16(128, DP, 1, 1);

  const int dq = 2 * (lane & 3);
  // the next row's index and CSR bounds are loaded one row ahead
  int64_t it = blockIdx.x;
  int64_t n_nx = 0, start_nx = 0, end_nx = 0;
  if (it < g.N) {
    n_nx = g.order ? (int64_t)g.order[it] : it;
    start_nx = g.rowptr[n_nx];
    end_nx = g.rowptr[n_nx + 1];
  }
  for (; it < g.N && alive; it += gridDim.x) {
    const int64_t n = n_nx, start = start_nx, end = end_nx;
    const int64_t it2 = it + gridDim.x;
    if (it2 < g.N) {
      n_nx = g.order ? (int64_t)g.order[it2] : it2;
      start_nx = g.rowptr[n_nx];
      end_nx = g.rowptr[n_nx + 1];
    }
    const float *xnp = g.X + (n + g.koff) * (int64_t)D;
    float xn[KG][2];
#pragma unroll
    for (int k = 0; k < KG; ++k) {
      const int d0 = 8 * k + dq;
      xn[k][0] = d0 < D ? xnp[d0] : 0.f;
      xn[k][1] = d0 + 1 < D ? xnp[d0 + 1] : 0.f;
    }
    float rsum = 0.f;
    bool bad = end < start;
    int ntile = 0;
    for (int64_t base = start; base < end; base += MT, ++ntile) {
      const int cnt = (int)((end - base) < MT ? (end - base) : MT);
      // gather: as in the E-step, warp w takes the 8-row batches w, w + 4,
      // w + 8, w + 12; lane l the row 8 b + l / 4 and the dimension pairs
      // 8 k + 2 (l % 4); all indices and weights, then all coordinates, are
      // loaded before any is used
      constexpr int NB = MT / 32;
      int32_t cb[NB];
      float rb[NB];
#pragma unroll
      for (int b = 0; b < NB; ++b) {
        const int p = 8 * (warp + 4 * b) + (lane >> 2);
        int32_t c = -1;
        float rv = 0.f;
        if (p < cnt) {
          c = g.col[base + p];
          rv = g.r[base + p];
          if (c < 0 || c >= g.npts) {
            bad = true;
            c = -1;
            rv = 0.f;
          }
        }
        cb[b] = c;
        rb[b] = rv;
      }
      float v[NB][KG][2];
#pragma unroll
      for (int b = 0; b < NB; ++b) {
        const float *xm = g.X + (int64_t)(cb[b] < 0 ? 0 : cb[b]) * D;
#pragma unroll
        for (int k = 0; k < KG; ++k) {
          const int d0 = 8 * k + dq;
          v[b][k][0] = (cb[b] >= 0 && d0 < D) ? xm[d0] : 0.f;
          v[b][k][1] = (cb[b] >= 0 && d0 + 1 < D) ? xm[d0 + 1] : 0.f;
        }
      }
#pragma unroll
      for (int b = 0; b < NB; ++b) {
        const int p = 8 * (warp + 4 * b) + (lane >> 2);
        if ((lane & 3) == 0) rsum += rb[b];
        const float w = sqrtf(rb[b] > 0.f ? rb[b] : 0.f);
#pragma unroll
        for (int k = 0; k < KG; ++k) {
          const int d0 = 8 * k + dq;
          const float x0 = cb[b] >= 0 ? w * (v[b][k][0] - xn[k][0]) : 0.f;
          const float x1 = cb[b] >= 0 ? w * (v[b][k][1] - xn[k][1]) : 0.f;
          uint32_t hi, lo;
          split2(x0, x1, hi, lo);
          *reinterpret_cast<uint32_t *>(G + core_off(p, d0, RS)) = hi;
          *reinterpret_cast<uint32_t *>(G + core_off(p, d0 + DP, RS)) = lo;
        }
      }
      fence_async_smem();
      fence_before();
      __syncthreads();
      if (tid == 0) {
        fence_after();
        const uint32_t g0 = smem_u32(G);
#pragma unroll
        for (int s = 0; s < MT / 16; ++s) {
          const uint32_t ko = 2 * s * LBO;
          const uint32_t acc = (ntile > 0 || s > 0) ? 1u : 0u;
          // [H; B] += [G_hi; G_lo]^T G_hi
          mma(tmem, desc(g0 + ko, LBO, SBO), desc(g0 + ko, LBO, SBO), idesc, acc);
        }
        commit(&mbar);
      }
      const bool ok = __syncthreads_and(mbar_wait(&mbar, phase) ? 1 : 0) != 0;
      phase ^= 1;
      fence_after();
      if (!ok) {
        if (tid == 0) atomicExch(g.err, 1);
        alive = false;
        break;
      }
      fence_before();
      __syncthreads();
    }
    if (!alive) break;
    // nu = nu0 + sum r (pairs in CSR order within warps, then warps)
    rsum = warp_sum(rsum);
    const bool any_bad = __syncthreads_or(bad ? 1 : 0);
    if (lane == 0) s_rs[warp] = rsum;
    // every thread copies its accumulator row (H row tid, or B row tid - 64)
    // to shared memory; then S_ij = H_ij + B_ij + B_ji
    const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll
    for (int c0 = 0; c0 < DP; c0 += 16) {
      float v1[16];
      if (end > start) {
        tmem_ld16(taddr + c0, v1);
      } else {
#pragma unroll
        for (int k = 0; k < 16; ++k) v1[k] = 0.f;
      }
#pragma unroll
      for (int k = 0; k < 16; k += 4)
        *reinterpret_cast<float4 *>(red + tid * RSTR + c0 + k) = make_float4(v1[k], v1[k + 1], v1[k + 2], v1[k + 3]);
    }
    __syncthreads();
    if (tid == 0) {
      const float nv = g.nu0 + (s_rs[0] + s_rs[1] + s_rs[2] + s_rs[3]);
      g.nu_out[n] = any_bad ? NAN : nv;
    }
    const float *H = red, *Bm = red + 64 * RSTR;
    if (g.SPo) {
      // tiled: warp w writes tiles w, w + 4, ... (256 contiguous bytes each),
      // zero outside D and above the diagonal
      float *dst = g.SPo + n * (int64_t)(g.ntile * 128);
      int t = 0;
      for (int I = 0; I < g.nt; ++I) {
        for (int J = 0; J <= I; ++J, ++t) {
          if ((t & 3) != warp) continue;
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int e = lane + 32 * h;
            const int i = 8 * I + (e >> 3), j = 8 * J + (e & 7);
            float v = 0.f;
            if (i < D && j <= i) v = (H[i * RSTR + j] + Bm[i * RSTR + j]) + Bm[j * RSTR + i];
            dst[t * 128 + e] = any_bad ? NAN : v;
          }
        }
      }
    } else {
      // coalesced stores: warp w writes rows w, w + 4, ..., lanes along the row
      float *Sn = g.S + n * (int64_t)D * D;
      for (int i = warp; i < D; i += 4) {
        const int jend = g.lower_only ? i + 1 : D;
        for (int j = lane; j < jend; j += 32)
          Sn[(int64_t)i * D + j] = any_bad ? NAN : (H[i * RSTR + j] + Bm[i * RSTR + j]) + Bm[j * RSTR + i];
      }
    }
    fence_before();
    __syncthreads();
  }
  __syncthreads();
  fence_after();
  if (warp == 0) tmem_dealloc(tmem, 64);
}

// ------------------------------------------------------- predictive density
// log p(y) = -log N + logsumexp_n [lc_n - h_n log1p(|W_triu_n^T (y - x_n)|^2)]
// (lakde/local_adaptive_kde.py:200-223) with the quad forms on the tensor
// cores: for each kernel n, the 128-query tiles of the query block are
// centred on x_n in fp32, split bf16 hi / lo (A) against W_triu_n hi / lo (B),
// 12 MMAs into tensor memory.  A CTA walks a chunk of kernels two at a time:
// each query tile is read once into registers and centred on both kernels;
// per query it keeps the running (max, sum) of its chunk in shared memory and
// writes it out as the chunk's partial at the end.  A second pass
// (pred_combine_kernel) folds the chunks.
constexpr int PQ = 4096;  // queries per block (one launch each)

struct PsmCfg {
  static constexpr uint32_t A_BYTES = MT * DP * 2;  // 16 KB
  static constexpr uint32_t B_BYTES = DP * DP * 2;  // 8 KB
  static constexpr uint32_t off_Ahi = 0, off_Alo = A_BYTES;
  static constexpr uint32_t off_B = 2 * A_BYTES;  // [kernel 0, 1][hi, lo]
  static constexpr uint32_t off_m = off_B + 4 * B_BYTES;
  static constexpr uint32_t off_s = off_m + PQ * 4;
  static constexpr uint32_t bytes = off_s + PQ * 4 + 128;
};

struct PredArgs {
  const float *X;
  const float *W;
  const float *lc;  // log coefficients [N]
  const float *nu;
  const float *Y;
  float *ws_m, *ws_s;  // [nchunks, Nq]
  int64_t N, Nq, q0, qn, chunk;
  int D;
  int *err;
};

__global__ void __launch_bounds__(128, 2) pred_tc_kernel(PredArgs g) {
  using C = PsmCfg;
  extern __shared__ __align__(128) unsigned char sm[];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t s_tmem;
  unsigned char *Ahi = sm + C::off_Ahi, *Alo = sm + C::off_Alo;
  float *pm = reinterpret_cast<float *>(sm + C::off_m);
  float *ps = reinterpret_cast<float *>(sm + C::off_s);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int D = g.D;
  const int dq = 2 * (lane & 3);

  if (warp == 0) tmem_alloc(&s_tmem, 128);
  if (tid == 0) mbar_init(&mbar);
  for (int i = tid; i < PQ; i += 128) {
    pm[i] = -INFINITY;
    ps[i] = 0.f;
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = s_tmem;
  uint32_t phase = 0;
  bool alive = true;
  constexpr uint32_t A_SBO = KG * 128, A_LBO = 128;
  constexpr uint32_t B_SBO = 128, B_LBO = KG * 128;
  const uint32_t idesc = idesc_bf16(MT, DP, 0, 1);
  const int64_t n_begin = (int64_t)blockIdx.x * g.chunk;
  const int64_t n_end = (n_begin + g.chunk < g.N) ? n_begin + g.chunk : g.N;
  const int ntiles = (int)((g.qn + MT - 1) / MT);

  for (int64_t n0 = n_begin; n0 < n_end && alive; n0 += 2) {
    const int nk = (n0 + 1 < n_end) ? 2 : 1;
    // W_triu of the kernels as B (hi, lo), their centres and coefficients
    float xn[2][KG][2], lc[2], hh[2];
#pragma unroll
    for (int kk = 0; kk < 2; ++kk) {
      const int64_t n = kk < nk ? n0 + kk : n0;
      const float *Wn = g.W + n * (int64_t)D * D;
      float wv[DP * DP / 256][2];
#pragma unroll
      for (int m = 0; m < DP * DP / 256; ++m) {
        const int e = tid + 128 * m;
        const int q = e >> 5, ln = e & 31;
        const int j = 8 * (q / KG) + (ln >> 2), i = 8 * (q % KG) + 2 * (ln & 3);
        wv[m][0] = (kk < nk && j < D && i < D) ? Wn[j * D + i] : 0.f;
        wv[m][1] = (kk < nk && j < D && i + 1 < D) ? Wn[j * D + i + 1] : 0.f;
      }
      const float *xp = g.X + n * (int64_t)D;
#pragma unroll
      for (int k = 0; k < KG; ++k) {
        const int d0 = 8 * k + dq;
        xn[kk][k][0] = d0 < D ? xp[d0] : 0.f;
        xn[kk][k][1] = d0 + 1 < D ? xp[d0 + 1] : 0.f;
      }
      lc[kk] = g.lc[n];
      hh[kk] = 0.5f * (g.nu[n] + 1.f);
      unsigned char *Bhi = sm + C::off_B + (2 * kk) * C::B_BYTES, *Blo = Bhi + C::B_BYTES;
#pragma unroll
      for (int m = 0; m < DP * DP / 256; ++m) {
        const int e = tid + 128 * m;
        const int q = e >> 5, ln = e & 31;
        const int j = 8 * (q / KG) + (ln >> 2), i = 8 * (q % KG) + 2 * (ln & 3);
        uint32_t hi, lo;
        split2(wv[m][0], wv[m][1], hi, lo);
        const uint32_t o = (uint32_t)(j >> 3) * B_LBO + (uint32_t)(i >> 3) * B_SBO + (uint32_t)(j & 7) * 16u +
                           (uint32_t)(i & 7) * 2u;
        *reinterpret_cast<uint32_t *>(Bhi + o) = hi;
        *reinterpret_cast<uint32_t *>(Blo + o) = lo;
      }
    }
    for (int t = 0; t < ntiles && alive; ++t) {
      // this thread's coordinates of the tile's queries (rows 8 (w + 4 b) + l / 4)
      constexpr int NB = MT / 32;
      float v[NB][KG][2];
      bool vq[NB];
#pragma unroll
      for (int b = 0; b < NB; ++b) {
        const int p = 8 * (warp + 4 * b) + (lane >> 2);
        const int64_t qi = (int64_t)t * MT + p;
        vq[b] = qi < g.qn;
        const float *yp = g.Y + (g.q0 + (vq[b] ? qi : 0)) * (int64_t)D;
#pragma unroll
        for (int k = 0; k < KG; ++k) {
          const int d0 = 8 * k + dq;
          v[b][k][0] = (vq[b] && d0 < D) ? yp[d0] : 0.f;
          v[b][k][1] = (vq[b] && d0 + 1 < D) ? yp[d0 + 1] : 0.f;
        }
      }
      for (int kk = 0; kk < nk; ++kk) {
#pragma unroll
        for (int b = 0; b < NB; ++b) {
          const int p = 8 * (warp + 4 * b) + (lane >> 2);
#pragma unroll
          for (int k = 0; k < KG; ++k) {
            const int d0 = 8 * k + dq;
            const float x0 = vq[b] ? v[b][k][0] - xn[kk][k][0] : 0.f;
            const float x1 = vq[b] ? v[b][k][1] - xn[kk][k][1] : 0.f;
            uint32_t hi, lo;
            split2(x0, x1, hi, lo);
            const uint32_t o = core_off(p, d0, A_SBO);
            *reinterpret_cast<uint32_t *>(Ahi + o) = hi;
            *reinterpret_cast<uint32_t *>(Alo + o) = lo;
          }
        }
        fence_async_smem();
        fence_before();
        __syncthreads();
        if (tid == 0) {
          fence_after();
          const uint32_t ahi = smem_u32(Ahi), alo = smem_u32(Alo);
          const uint32_t bhi = smem_u32(sm + C::off_B + (2 * kk) * C::B_BYTES), blo = bhi + C::B_BYTES;
          const uint32_t td = tmem + 64u * (uint32_t)kk;
#pragma unroll
          for (int s = 0; s < DP / 16; ++s) {
            const uint32_t ao = 2 * s * A_LBO, bo = 2 * s * B_LBO;
            mma(td, desc(ahi + ao, A_LBO, A_SBO), desc(bhi + bo, B_LBO, B_SBO), idesc, s > 0);
            mma(td, desc(alo + ao, A_LBO, A_SBO), desc(bhi + bo, B_LBO, B_SBO), idesc, 1);
            mma(td, desc(ahi + ao, A_LBO, A_SBO), desc(blo + bo, B_LBO, B_SBO), idesc, 1);
          }
          commit(&mbar);
        }
        // A is rewritten for the next kernel only after these MMAs completed
        const bool ok = __syncthreads_and(mbar_wait(&mbar, phase) ? 1 : 0) != 0;
        phase ^= 1;
        fence_after();
        if (!ok) {
          if (tid == 0) atomicExch(g.err, 1);
          alive = false;
          break;
        }
      }
      if (!alive) break;
      // epilogue: thread = query row; fold the kernels into the running
      // (max, sum) of the query
      const int64_t qi = (int64_t)t * MT + tid;
      const uint32_t lane_base = (uint32_t)(warp * 32) << 16;
      for (int kk = 0; kk < nk; ++kk) {
        float q = 0.f;
#pragma unroll
        for (int c0 = 0; c0 < DP; c0 += 16) {
          float vv[16];
          tmem_ld16(tmem + lane_base + 64u * (uint32_t)kk + c0, vv);
#pragma unroll
          for (int k = 0; k < 16; ++k) q = fmaf(vv[k], vv[k], q);
        }
        if (qi < g.qn) {
          // hardware log and exp: a few 1e-5 nats at most on the density
          const float lp = lc[kk] - hh[kk] * __logf(1.f + q);
          const float m = pm[qi];
          if (lp > m) {
            ps[qi] = ps[qi] * __expf(m - lp) + 1.f;
            pm[qi] = lp;
          } else {
            ps[qi] += __expf(lp - m);
          }
        }
      }
      fence_before();
      __syncthreads();
    }
  }
  __syncthreads();
  // this chunk's partials for the query block
  for (int64_t i = tid; i < g.qn; i += 128) {
    g.ws_m[(int64_t)blockIdx.x * g.Nq + g.q0 + i] = pm[i];
    g.ws_s[(int64_t)blockIdx.x * g.Nq + g.q0 + i] = ps[i];
  }
  fence_after();
  if (warp == 0) tmem_dealloc(tmem, 128);
}

// out[q] = -log N + logsumexp over the chunks' (max, sum) partials
__global__ void pred_fold_kernel(const float *__restrict__ ws_m, const float *__restrict__ ws_s,
                                 float *__restrict__ out, int64_t Nq, int64_t nchunks, float log_n) {
  const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (q >= Nq) return;
  float M = -INFINITY;
  for (int64_t c = 0; c < nchunks; ++c) M = fmaxf(M, ws_m[c * Nq + q]);
  float S = 0.f;
  if (M != -INFINITY)
    for (int64_t c = 0; c < nchunks; ++c) S += ws_s[c * Nq + q] * expf(ws_m[c * Nq + q] - M);
  out[q] = (M == -INFINITY) ? M : (M + logf(S)) - log_n;
}

}  // namespace tc
}  // namespace lakde

using namespace lakde;

static int tc_common_checks(const char *what, int dtype, int64_t N, int64_t D, int64_t npts, int64_t koff) {
  if (dtype != LAKDE_F32) {
    set_error("%s: float32 values only", what);
    return LAKDE_EDTYPE;
  }
  if (N < 0 || D < 1 || koff < 0 || npts < N + koff) {
    set_error("%s: invalid sizes", what);
    return LAKDE_EINVAL;
  }
  if (D > 64) {
    set_error("%s: D=%lld exceeds 64", what, (long long)D);
    return LAKDE_EUNSUPPORTED;
  }
  return LAKDE_OK;
}

// Persistent grid: the CTAs that are resident at once, limited by shared
// memory (228 KB per SM, 1 KB reserved per CTA), tensor memory (512 columns
// per SM) and registers (64 K per SM), so that no CTA waits for a second wave.
template <typename Kern>
static int tc_grid(Kern kern, size_t smem, int tmem_cols, int64_t N, unsigned *grid) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1) sms = 148;
  int per_sm = (int)((228u * 1024u) / (smem + 1024u + 512u));
  if (per_sm > 512 / tmem_cols) per_sm = 512 / tmem_cols;
  cudaFuncAttributes fa;
  if (cudaFuncGetAttributes(&fa, kern) == cudaSuccess && fa.numRegs > 0) {
    const int regs_warp = ((fa.numRegs * 32 + 255) / 256) * 256;  // allocated per warp in units of 256
    const int by_regs = 65536 / (4 * regs_warp);
    if (per_sm > by_regs) per_sm = by_regs;
  }
  if (per_sm > 8) per_sm = 8;
  if (per_sm < 1) per_sm = 1;
  int64_t g = (int64_t)sms * per_sm;
  if (g > N) g = N;
  *grid = (unsigned)(g < 1 ? 1 : g);
  return LAKDE_OK;
}

extern "C" int lakde_estep_tc(int dtype, int64_t N, int64_t D, int64_t npts, const void *rowptr, const void *col,
                              const void *order, const void *X, int64_t kernel_offset, const void *W_triu,
                              const void *nu, const void *logdet_W, void *logrho, int32_t *err, void *stream) {
  clear_error();
  if (int st = tc_common_checks("estep_tc", dtype, N, D, npts, kernel_offset)) return st;
  if (N == 0) return LAKDE_OK;
  if (!rowptr || !col || !X || !W_triu || !nu || !logdet_W || !logrho || !err) {
    set_error("estep_tc: null pointer");
    return LAKDE_EINVAL;
  }
  if (int st = bind_device("estep_tc", {logrho, rowptr, col, order, X, W_triu, nu, logdet_W, err})) return st;
  tc::TcArgs g{};
  g.rowptr = static_cast<const int64_t *>(rowptr);
  g.col = static_cast<const int32_t *>(col);
  g.order = static_cast<const int32_t *>(order);
  g.X = static_cast<const float *>(X);
  g.W = static_cast<const float *>(W_triu);
  g.nu = static_cast<const float *>(nu);
  g.logdet = static_cast<const float *>(logdet_W);
  g.logrho = static_cast<float *>(logrho);
  g.npts = npts;
  g.koff = kernel_offset;
  g.N = N;
  g.D = (int)D;
  g.err = err;
  const size_t smem = tc::EsmCfg::bytes;
  cudaError_t e = cudaFuncSetAttribute(tc::estep_tc_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) {
    set_error("estep_tc: %s", cudaGetErrorString(e));
    return LAKDE_ECUDA;
  }
  unsigned grid;
  tc_grid(tc::estep_tc_kernel<false>, smem, 64, N, &grid);
  tc::estep_tc_kernel<false><<<grid, 128, smem, as_stream(stream)>>>(g);
  return check_launch("estep_tc");
}

extern "C" int lakde_mstep_tc(int dtype, int64_t N, int64_t D, int64_t npts, const void *rowptr, const void *col,
                              const void *order, const void *r, const void *X, int64_t kernel_offset, double nu_0,
                              void *S, void *nu, int lower_only, int32_t *err, void *stream) {
  clear_error();
  if (int st = tc_common_checks("mstep_tc", dtype, N, D, npts, kernel_offset)) return st;
  if (N == 0) return LAKDE_OK;
  if (!rowptr || !col || !r || !X || !S || !nu || !err) {
    set_error("mstep_tc: null pointer");
    return LAKDE_EINVAL;
  }
  if (int st = bind_device("mstep_tc", {S, rowptr, col, order, r, X, nu, err})) return st;
  tc::TcArgs g{};
  g.rowptr = static_cast<const int64_t *>(rowptr);
  g.col = static_cast<const int32_t *>(col);
  g.order = static_cast<const int32_t *>(order);
  g.r = static_cast<const float *>(r);
  g.X = static_cast<const float *>(X);
  g.S = static_cast<float *>(S);
  g.nu_out = static_cast<float *>(nu);
  g.nu0 = (float)nu_0;
  g.lower_only = lower_only != 0;
  g.npts = npts;
  g.koff = kernel_offset;
  g.N = N;
  g.D = (int)D;
  g.err = err;
  const size_t smem = tc::MsmCfg::bytes;
  cudaError_t e = cudaFuncSetAttribute(tc::mstep_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) {
    set_error("mstep_tc: %s", cudaGetErrorString(e));
    return LAKDE_ECUDA;
  }
  unsigned grid;
  tc_grid(tc::mstep_tc_kernel, smem, 64, N, &grid);
  tc::mstep_tc_kernel<<<grid, 128, smem, as_stream(stream)>>>(g);
  return check_launch("mstep_tc");
}

static int64_t pred_tc_chunks(int64_t N) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1) sms = 148;
  int64_t nchunks = 2 * (int64_t)sms;  // two CTAs per SM (shared memory, TMEM)
  if (nchunks > (N + 1) / 2) nchunks = (N + 1) / 2;
  return nchunks < 1 ? 1 : nchunks;
}

extern "C" size_t lakde_log_pred_density_tc_workspace(int64_t N, int64_t Nq, int64_t D) {
  if (N <= 0 || Nq <= 0 || D < 1 || D > 64) return 0;
  return (size_t)(2 * pred_tc_chunks(N) * Nq) * sizeof(float);
}

extern "C" int lakde_log_pred_density_tc(int dtype, int64_t N, int64_t Nq, int64_t D, const void *X,
                                         const void *W_triu, const void *nu, const void *log_coeff, const void *Y,
                                         void *out, void *workspace, size_t workspace_bytes, int32_t *err,
                                         void *stream) {
  clear_error();
  if (dtype != LAKDE_F32) {
    set_error("log_pred_density_tc: float32 values only");
    return LAKDE_EDTYPE;
  }
  if (N < 1 || Nq < 0 || D < 1 || D > 64) {
    set_error("log_pred_density_tc: invalid sizes (N=%lld, Nq=%lld, D=%lld)", (long long)N, (long long)Nq,
              (long long)D);
    return D > 64 ? LAKDE_EUNSUPPORTED : LAKDE_EINVAL;
  }
  if (Nq == 0) return LAKDE_OK;
  const size_t need = lakde_log_pred_density_tc_workspace(N, Nq, D);
  if (!workspace || workspace_bytes < need) {
    set_error("log_pred_density_tc: workspace of %zu bytes needed, %zu given", need, workspace_bytes);
    return LAKDE_EINVAL;
  }
  if (!X || !W_triu || !nu || !log_coeff || !Y || !out || !err) {
    set_error("log_pred_density_tc: null pointer");
    return LAKDE_EINVAL;
  }
  if (int st = bind_device("log_pred_density_tc", {out, X, W_triu, nu, log_coeff, Y, workspace, err})) return st;
  const int64_t nchunks = pred_tc_chunks(N);
  tc::PredArgs g{};
  g.X = static_cast<const float *>(X);
  g.W = static_cast<const float *>(W_triu);
  g.lc = static_cast<const float *>(log_coeff);
  g.nu = static_cast<const float *>(nu);
  g.Y = static_cast<const float *>(Y);
  g.ws_m = static_cast<float *>(workspace);
  g.ws_s = g.ws_m + nchunks * Nq;
  g.N = N;
  g.Nq = Nq;
  g.chunk = (N + nchunks - 1) / nchunks;
  g.D = (int)D;
  g.err = err;
  const size_t smem = tc::PsmCfg::bytes;
  cudaError_t e = cudaFuncSetAttribute(tc::pred_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) {
    set_error("log_pred_density_tc: %s", cudaGetErrorString(e));
    return LAKDE_ECUDA;
  }
  const int64_t grid = (N + g.chunk - 1) / g.chunk;
  for (int64_t q0 = 0; q0 < Nq; q0 += tc::PQ) {
    g.q0 = q0;
    g.qn = (Nq - q0) < tc::PQ ? (Nq - q0) : tc::PQ;
    tc::pred_tc_kernel<<<(unsigned)grid, 128, smem, as_stream(stream)>>>(g);
    if (int st = check_launch("log_pred_density_tc")) return st;
  }
  tc::pred_fold_kernel<<<(unsigned)((Nq + 255) / 256), 256, 0, as_stream(stream)>>>(
      g.ws_m, g.ws_s, static_cast<float *>(out), Nq, grid, (float)log((double)N));
  return check_launch("log_pred_density_tc_combine");
}

extern "C" int64_t lakde_tile_count(int64_t D);

extern "C" int lakde_mstep_tc_tiled(int dtype, int64_t N, int64_t D, int64_t npts, const void *rowptr,
                                    const void *col, const void *order, const void *r, const void *X,
                                    int64_t kernel_offset, double nu_0, void *SP, void *nu, int32_t *err,
                                    void *stream) {
  clear_error();
  if (int st = tc_common_checks("mstep_tc_tiled", dtype, N, D, npts, kernel_offset)) return st;
  if (D <= 8) {
    set_error("mstep_tc_tiled: needs 8 < D <= 64");
    return LAKDE_EUNSUPPORTED;
  }
  if (N == 0) return LAKDE_OK;
  if (!rowptr || !col || !r || !X || !SP || !nu || !err) {
    set_error("mstep_tc_tiled: null pointer");
    return LAKDE_EINVAL;
  }
  if (int st = bind_device("mstep_tc_tiled", {SP, rowptr, col, order, r, X, nu, err})) return st;
  tc::TcArgs g{};
  g.rowptr = static_cast<const int64_t *>(rowptr);
  g.col = static_cast<const int32_t *>(col);
  g.order = static_cast<const int32_t *>(order);
  g.r = static_cast<const float *>(r);
  g.X = static_cast<const float *>(X);
  g.SPo = static_cast<float *>(SP);
  g.ntile = (int)lakde_tile_count(D);
  while ((g.nt + 1) * (g.nt + 2) / 2 <= g.ntile) ++g.nt;
  g.nu_out = static_cast<float *>(nu);
  g.nu0 = (float)nu_0;
  g.npts = npts;
  g.N = N;
  g.koff = kernel_offset;
  g.D = (int)D;
  g.err = err;
  const size_t smem = tc::MsmCfg::bytes;
  cudaError_t e = cudaFuncSetAttribute(tc::mstep_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) {
    set_error("mstep_tc_tiled: %s", cudaGetErrorString(e));
    return LAKDE_ECUDA;
  }
  unsigned grid;
  tc_grid(tc::mstep_tc_kernel, smem, 64, N, &grid);
  tc::mstep_tc_kernel<<<grid, 128, smem, as_stream(stream)>>>(g);
  return check_launch("mstep_tc_tiled");
}

extern "C" int lakde_estep_tc_tiled(int dtype, int64_t N, int64_t D, int64_t npts, const void *rowptr,
                                    const void *col, const void *order, const void *X, int64_t kernel_offset,
                                    const void *W_cores, const void *nu, const void *logdet_W, void *logrho,
                                    int32_t *err, void *stream) {
  clear_error();
  if (int st = tc_common_checks("estep_tc_tiled", dtype, N, D, npts, kernel_offset)) return st;
  if (D <= 8) {
    set_error("estep_tc_tiled: needs 8 < D <= 64");
    return LAKDE_EUNSUPPORTED;
  }
  if (N == 0) return LAKDE_OK;
  if (!rowptr || !col || !X || !W_cores || !nu || !logdet_W || !logrho || !err) {
    set_error("estep_tc_tiled: null pointer");
    return LAKDE_EINVAL;
  }
  if (reinterpret_cast<uintptr_t>(W_cores) & 15u) {
    set_error("estep_tc_tiled: W_cores must be 16-byte aligned");
    return LAKDE_EINVAL;
  }
  if (int st = bind_device("estep_tc_tiled", {logrho, rowptr, col, order, X, W_cores, nu, logdet_W, err})) return st;
  tc::TcArgs g{};
  g.rowptr = static_cast<const int64_t *>(rowptr);
  g.col = static_cast<const int32_t *>(col);
  g.order = static_cast<const int32_t *>(order);
  g.X = static_cast<const float *>(X);
  g.Wc = static_cast<const uint32_t *>(W_cores);
  g.ntile = (int)lakde_tile_count(D);
  while ((g.nt + 1) * (g.nt + 2) / 2 <= g.ntile) ++g.nt;
  g.nu = static_cast<const float *>(nu);
  g.logdet = static_cast<const float *>(logdet_W);
  g.logrho = static_cast<float *>(logrho);
  g.npts = npts;
  g.N = N;
  g.koff = kernel_offset;
  g.D = (int)D;
  g.err = err;
  const size_t smem = tc::EsmCfg::bytes;
  cudaError_t e = cudaFuncSetAttribute(tc::estep_tc_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) {
    set_error("estep_tc_tiled: %s", cudaGetErrorString(e));
    return LAKDE_ECUDA;
  }
  unsigned grid;
  tc_grid(tc::estep_tc_kernel<true>, smem, 64, N, &grid);
  tc::estep_tc_kernel<true><<<grid, 128, smem, as_stream(stream)>>>(g);
  return check_launch("estep_tc_tiled");
}
