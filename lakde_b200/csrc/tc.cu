// Mixed-precision tensor-core (tcgen05, kind::tf32) kernels of the large-D VI
// path and of the predictive density.
//
// Grouping pairs by kernel makes two dense contractions per kernel row n with
// m_n pairs, Delta = [x_m - x_n] (m_n x D):
//   E-step  Y = Delta W_triu_n  (m_n x D),  Q_p = |Y_p|^2           (lakde/local_adaptive_kde.py:36-44)
//   M-step  S_n = G^T G,  G = sqrt(r) Delta                          (lakde/local_adaptive_kde.py:66-81)
// and log_pred_density is the E-step contraction with every query of a block
// as the "pairs" of every kernel (lakde/local_adaptive_kde.py:200-223).
//
// Precision: the differences are centred on the kernel in fp32 and split as
// x = hi + lo with hi = tf32(x) and lo = tf32(x - hi) (round to nearest; 11 +
// 11 significant bits, |lo| <= 2^-11 |x|), with fp32 accumulation in tensor
// memory.  The M-step forms all four blocks of (G_hi + G_lo)^T (G_hi + G_lo):
// dropping lo*lo there would take a positive semi-definite 2^-24-relative
// term off S, which shrinks exactly the small eigenvalues of a near-singular
// neighbourhood.  The E-step likewise forms all four products of
// (D_hi + D_lo) (W_hi + W_lo) (two MMAs per K step against [W_hi | W_lo]);
// what remains is the rounding of lo, below 2^-22 relative with random sign.
//
// One persistent CTA per SM, 384 threads in four roles, pipelined over
// 128-pair tiles with mbarriers:
//   * a metadata warp takes kernel rows 32 at a time (an atomic row queue
//     over the caller's longest-first order, or a static stride), one lane
//     per row for the dependent loads and the E-step's digamma sums, and
//     writes each tile's row, pair range, column indices and weights into a
//     ring of 8 slots, loading the next tile's indices while it writes one;
//   * two gather warps copy each tile's pair rows (rows of X padded to a
//     multiple of 16 bytes) into one of two raw stages with cp.async, the
//     first also its kernel centre and, for the first tile of a row, the row's
//     W cores into one of two B stages by bulk copy, after the stage's last
//     MMAs committed;
//   * 8 consumer warps convert tile t (centre, M-step: scale by sqrt r, split
//     into the hi / lo core-matrix tile) and read the previous tile's
//     accumulator (one TMEM lane per pair) to write log rho / S_n / the
//     running log-sum-exp;
//   * an MMA warp issues each converted tile's MMAs into one of two TMEM
//     accumulators and commits them to mbarriers.
// Every wait is bounded: on a time-out the kernel sets *err, waits (bounded)
// for its own copies and MMAs in flight, frees its TMEM and returns.
//
// Shared-memory operand layout (canonical, no swizzle; a core matrix is 8 rows
// x 16 bytes = 8 x 4 tf32):
//   tile   E-step / predictive density: 16 pair groups x 32 cores: core
//          c < 16 holds dims 4c..4c+3 of the 8 pairs' hi parts, core 16 + c
//          the lo parts; the A operand (K-major, M = pairs): LBO = 128 (next
//          4 dims), SBO = 4096 (next 8 pairs).
//          M-step: G^T, rows = [hi dims 0..63; lo dims 0..63], K = pairs:
//          core (row group r / 8, pair quad p / 4) at (r / 8) GT_SBO +
//          (p / 4) 128; A = [G_hi; G_lo]^T (M = 128) and B = G_hi (its first
//          N rows) are both K-major with LBO = 128 (next 4 pairs) and SBO =
//          GT_SBO (next 8 rows); GT_SBO = 4112 rather than 4096 keeps the
//          converters' 16-byte stores on distinct bank groups.
//   B      W cores (K-major, N = output dim i, K = input dim j, element (i, j)
//          = W_triu[j][i] = X[i][j] with X = L^-1 lower): per K step J the
//          2 DP / 8 row groups of 2 cores each, the hi parts of output
//          blocks I = 0..DP/8-1 then their lo parts; LBO = 128, SBO = 256,
//          N = 2 DP.
#include "common.cuh"

namespace lakde {
namespace tc {

constexpr int MT = 128;        // pairs (queries) per tile: the MMA M
constexpr int NTHR = 256;      // 8 consumer warps (two more produce)
constexpr int NS = 8;          // metadata slots
constexpr int NGW = 2;         // gather warps (four measured no faster: the scattered copies, not their issue, set the rate)
constexpr int RAW_STRIDE = 272;  // bytes per staged pair row: 64 floats + 16 bytes against bank conflicts
constexpr uint32_t kSpinLimit = 1u << 26;
constexpr uint64_t kWaitLimitNs = 1500000000ull;  // 1.5 s: far above any copy or MMA of one tile
constexpr int PQ = 2048;       // queries per predictive-density launch
constexpr uint32_t GT_SBO = 4112;  // M-step tile: bytes between 8-row groups of G^T

enum Mode { ESTEP = 0, MSTEP = 1, PRED = 2 };

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor: no swizzle, version 1 (sm_100).
__device__ __forceinline__ uint64_t desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | ((uint64_t)1 << 46);
}

// Instruction descriptor, kind::tf32: tf32 x tf32 -> f32, M x N, operand majors
// (0 = K-major, 1 = MN-major).
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int N, int a_mn_major, int b_mn_major) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)a_mn_major << 15) | ((uint32_t)b_mn_major << 16) |
         ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void commit(uint64_t *mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(mbar))
               : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t *mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *mbar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(mbar)) : "memory");
}

__device__ __forceinline__ void mbar_arrive_tx(uint64_t *mbar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(mbar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Waits for the phase with the given parity; false once kWaitLimitNs have
// passed (checked every 1024 polls) or after kSpinLimit polls.
__device__ __forceinline__ bool mbar_wait(uint64_t *mbar, uint32_t parity) {
  const uint32_t addr = smem_u32(mbar);
  uint64_t t0 = 0;
  for (uint32_t it = 0; it < kSpinLimit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(addr), "r"(parity)
        : "memory");
    if (done) return true;
    if ((it & 1023u) == 0) {
      const uint64_t now = global_ns();
      if (it == 0) t0 = now;
      else if (now - t0 > kWaitLimitNs) return false;
    }
  }
  return false;
}

// Global -> shared bulk copy completing on mbar (16-byte aligned addresses, size a multiple of 16).
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void *src, uint32_t bytes, uint64_t *mbar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(smem_u32(mbar))
               : "memory");
}

__device__ __forceinline__ void prefetch_l2(const void *src, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
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

// 16 consecutive fp32 columns at each of two TMEM addresses of this thread's
// lane, one wait for both.
__device__ __forceinline__ void tmem_ld16x2(uint32_t ta, uint32_t tb, float (&v)[16], float (&u)[16]) {
  uint32_t r[16], q[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(ta));
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];\n"
      : "=r"(q[0]), "=r"(q[1]), "=r"(q[2]), "=r"(q[3]), "=r"(q[4]), "=r"(q[5]), "=r"(q[6]), "=r"(q[7]),
        "=r"(q[8]), "=r"(q[9]), "=r"(q[10]), "=r"(q[11]), "=r"(q[12]), "=r"(q[13]), "=r"(q[14]), "=r"(q[15])
      : "r"(tb));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    v[i] = __uint_as_float(r[i]);
    u[i] = __uint_as_float(q[i]);
  }
}

__device__ __forceinline__ void split4(const float4 x, float4 &hi, float4 &lo) {
  hi = make_float4(tf32_rna(x.x), tf32_rna(x.y), tf32_rna(x.z), tf32_rna(x.w));
  lo = make_float4(tf32_rna(x.x - hi.x), tf32_rna(x.y - hi.y), tf32_rna(x.z - hi.z), tf32_rna(x.w - hi.w));
}

// Float offset of segment J of a W-core block (segments J' < J hold NT - J'
// hi tiles then as many lo tiles, 64 floats each).
__host__ __device__ constexpr int wseg(int J, int NT) { return 128 * (J * NT - J * (J - 1) / 2); }

struct Args {
  const int64_t *rowptr;
  const int32_t *col;
  const int32_t *order;
  const float *r;        // M-step weights
  const float *X;        // kernel centres (and the pair points of the E- and M-step), row stride ldx
  int64_t ldx;
  const float *Y;        // predictive density: queries, row stride ldy
  int64_t ldy;
  const float *Wc;       // E-step / predictive density: W cores, ntile * 64 floats per kernel
  const float *nu;       // E-step: nu_n; predictive density: nu_n
  const float *logdet;   // E-step
  const float *lc;       // predictive density: log coefficient per kernel
  float *logrho;         // E-step output, CSR order
  float *S;              // M-step output [N, D, D] (dense) ...
  int lower_only;
  float *SPo;            // ... or the S halves of the interleaved S / P tiles
  float *nu_out;         // M-step output
  float nu0;
  float *ws_m, *ws_s;    // predictive density partials [gridDim.x, Nq]
  int64_t Nq, q0, qn, chunk;
  int64_t npts;          // rows of X (pair points) or of Y (queries)
  int64_t N;
  int64_t koff;          // row n is the kernel centred on X[n + koff]
  int D;
  int nt;                // 8-row blocks of the tiled layouts (W cores, SP)
  int ntile;             // nt (nt + 1) / 2
  int32_t *queue;        // row counter of the work queue (zero at launch), or null
  int32_t *err;
  int stall;             // test hook: the first stage expects 16 bytes no copy delivers
};

// Shared memory of one CTA.  The E-step and the predictive density keep two
// A tiles that take the gathered pair rows in place (the MMAs of one tile
// run while the other is converted); the M-step transposes, so its rows
// land in two raw stages and it converts into one tile.  The B stages of
// the E-step / predictive density are the accumulator copy of the M-step's
// epilogue.
template <int MODE>
struct SmemL {
  static constexpr bool DUAL = MODE != MSTEP;
  static constexpr uint32_t TILE_BYTES = DUAL ? 65536u : 16u * GT_SBO;   // M-step: 16 x GT_SBO
  static constexpr uint32_t TILE = 0;                                   // 2 (M-step: 1) A tiles
  static constexpr uint32_t RAW = TILE + (DUAL ? 2 : 1) * TILE_BYTES;   // M-step: 2 x 34 KB
  static constexpr uint32_t BST = RAW + (DUAL ? 0 : 2 * MT * RAW_STRIDE);  // 2 x (hi 16 KB + lo 16 KB)
  static constexpr uint32_t B_BYTES = 16384;
  static constexpr uint32_t RSTR = 68;                                  // M-step accumulator copy row stride
  static constexpr uint32_t RED = BST;
  static constexpr uint32_t XN = BST + 4 * B_BYTES;                     // NS x 256 B kernel centres
  static constexpr uint32_t CIDX = XN + NS * 256;                       // NS x 128 int
  static constexpr uint32_t RV = CIDX + NS * MT * 4;                    // NS x 128 float
  static constexpr uint32_t META = RV + NS * MT * 4;                    // NS x Meta
  static constexpr uint32_t PM = META + NS * 64;                        // predictive density (max, sum)
  static constexpr uint32_t BAR = PM + 2 * PQ * 4;                      // mbarriers
  static constexpr uint32_t bytes = BAR + 256;
};
static_assert(SmemL<MSTEP>::RSTR * 128 * 4 <= 4 * SmemL<MSTEP>::B_BYTES, "accumulator copy fits the B stages");
static_assert(SmemL<MSTEP>::bytes + 1024 <= 232448 && SmemL<ESTEP>::bytes + 1024 <= 232448,
              "shared memory of one CTA");

// mbarriers (8 bytes each from SmemL::BAR)
struct Bars {
  static constexpr int MFULL = 0;          // [NS] metadata of a slot written (32 producer lanes)
  static constexpr int MEMPTY = NS;        // [NS] slot free again (consumer thread 0)
  static constexpr int RFULL = 2 * NS;     // [2] pair rows and kernel centre landed (64 gatherer lanes + 1)
  static constexpr int REMPTY = RFULL + 2; // [2] rows' buffer free: M-step raw stage converted, else A tile's MMAs done
  static constexpr int BFULL = REMPTY + 2; // [2] W cores of a B stage landed
  static constexpr int BEMPTY = BFULL + 2; // [2] MMAs of the stage's last row done (tcgen05.commit)
  static constexpr int MMA = BEMPTY + 2;   // [2] MMAs of tile t done (t % 2; tcgen05.commit)
  static constexpr int CONV = MMA + 2;     // [2] tile t converted (t % 2; every consumer thread)
  static constexpr int COUNT = CONV + 2;
};
static_assert(Bars::COUNT * 8 <= 256, "mbarrier area");

struct Meta {
  int64_t n;      // kernel row (< 0: no more tiles)
  int64_t base;   // first pair of the tile (CSR position; predictive density: query offset in the block)
  int cnt;        // pairs in the tile
  int flags;      // 1: first tile of its row, 2: last tile, 4: row has an invalid index, 8: B stage used before
  int bs;         // B stage / accumulator of the row (row counter parity)
  int bph;        // parity of this row's use of B stage bs (its W-copy mbarrier phase)
  float c0, c1;   // E-step: 0.5 E[log|Lambda|], -nu / 2;  predictive density: log coefficient, (nu + 1) / 2
  float rsum;     // M-step: sum of r over the row (last tile)
};

// All 32 lanes of a warp AND-reduce v over the n threads of named barrier id.
__device__ __forceinline__ bool bar_and(int id, int n, bool v) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\tsetp.ne.u32 p, %1, 0;\n\tbar.red.and.pred q, %2, %3, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}\n"
      : "=r"(r)
      : "r"((uint32_t)v), "r"(id), "r"(n)
      : "memory");
  return r != 0;
}

__device__ __forceinline__ void bar_sync(int id, int n) { asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory"); }

template <int MODE, int DP>
struct Kern {
  using Smem = SmemL<MODE>;
  static constexpr int NCH = DP / 4;     // 4-dim chunks of a row
  static constexpr int HCH = NCH / 2;    // chunks per converter thread
  // M-step accumulator columns: the hi rows 0..63 of G^T, then its lo rows
  // 64..64 + DP (rounded up to 16, the MMA's N granule)
  static constexpr int MN = 64 + ((DP + 15) / 16) * 16;
  // TMEM columns of one accumulator (two are allocated): the M-step's
  // [hi | lo] rows of G^T, the E-step's [hi | lo] output columns
  static constexpr uint32_t ACC_COLS = 128u;
  static constexpr int NG = DP / 8;  // 8-row groups of one half of a B stage's K step

  // ------------------------------------------------------- metadata warp
  // State of the metadata warp.  Rows are fetched 32 at a time, lane j
  // holding row j of the batch (its index, pair range and row constants:
  // the dependent loads and the digamma sums of 32 rows run side by side);
  // tiles are planned from the batch, and each tile's column indices and
  // weights are loaded one tile before they are written.
  struct Prod {
    int64_t bn, ba, bb;  // this lane's batch row: kernel (-1: none) and pair range
    float bc0, bc1;      // its row constants
    int bsz, bidx;       // rows in the batch, next one to start
    int64_t popped;      // row slots taken by this CTA
    bool exhausted;      // no rows left to fetch
    bool done;
    int64_t n, next, end;  // current row and the first pair of its next tile
    int rows;            // rows started (their parity selects the B stage / accumulator)
    int bpar, bused;     // bit b: parity of the next use of B stage b, stage b used
    float c0, c1;
    int rowbad;          // the current row's pair range is invalid
    float racc;          // M-step: running sum of r over the row (at write time)
    int bad;             // M-step: invalid index seen in the row (at write time)
  };

  struct Plan {
    int64_t n, base;
    int cnt, flags, bs, bph;
    float c0, c1;
  };

  // The next 32 row slots of this CTA: the work queue (an atomic counter
  // over the caller's row order, 32 slots per claim), a static stride over
  // the grid without a queue, or the CTA's contiguous chunk of kernels for the
  // predictive density.  Valid slots are a prefix of the lanes.
  static __device__ void fetch_batch(const Args &g, Prod &P, int lane) {
    int64_t it;
    bool valid = true;
    if (MODE == PRED) {
      valid = P.popped + lane < g.chunk;
      it = (int64_t)blockIdx.x * g.chunk + P.popped + lane;
    } else if (g.queue) {
      int v = 0;
      if (lane == 0) v = atomicAdd(g.queue, 32);
      it = (int64_t)__shfl_sync(0xffffffffu, v, 0) + lane;
    } else {
      it = (int64_t)blockIdx.x + (P.popped + lane) * (int64_t)gridDim.x;
    }
    P.popped += 32;
    valid = valid && it < g.N;
    int64_t n = -1, a = 0, b = 0;
    float c0 = 0.f, c1 = 0.f;
    if (valid) {
      n = (MODE != PRED && g.order) ? (int64_t)g.order[it] : it;
      if (MODE != PRED) {
        a = g.rowptr[n];
        b = g.rowptr[n + 1];
      } else {
        b = g.qn;
      }
      if (MODE == ESTEP) {
        // 0.5 (psi_D(nu / 2) + D log 2 + logdet W), -nu / 2
        const float nv = g.nu[n];
        const float ld = g.logdet[n];
        double md = 0.0;
        for (int i = 1; i <= g.D; ++i) md += digamma_d(0.5 * (double)nv + 0.5 * (1 - i));
        c0 = (float)(0.5 * (md + g.D * 0.69314718055994530942 + (double)ld));
        c1 = -0.5f * nv;
      } else if (MODE == PRED) {
        c0 = g.lc[n];
        c1 = 0.5f * (g.nu[n] + 1.f);
      }
    }
    P.bn = n;
    P.ba = a;
    P.bb = b;
    P.bc0 = c0;
    P.bc1 = c1;
    P.bsz = __popc(__ballot_sync(0xffffffffu, valid));
    P.bidx = 0;
    if (P.bsz < 32) P.exhausted = true;
  }

  // Plans the next tile (n < 0: no work left).
  static __device__ Plan plan_tile(const Args &g, Prod &P, int lane) {
    Plan t{};
    bool first = false;
    if (!P.done && P.next >= P.end) {
      for (;;) {
        if (P.bidx >= P.bsz) {
          if (P.exhausted) {
            P.done = true;
            break;
          }
          fetch_batch(g, P, lane);
          continue;
        }
        const int j = P.bidx++;
        const int64_t n = __shfl_sync(0xffffffffu, P.bn, j);
        const int64_t a = __shfl_sync(0xffffffffu, P.ba, j);
        const int64_t b = __shfl_sync(0xffffffffu, P.bb, j);
        const float c0 = __shfl_sync(0xffffffffu, P.bc0, j);
        const float c1 = __shfl_sync(0xffffffffu, P.bc1, j);
        if (MODE == ESTEP && b <= a) continue;  // no pairs: no log rho to write
        P.n = n;
        P.next = a;
        P.end = b < a ? a : b;  // an M-step row without pairs still gets one (empty) tile
        P.rowbad = b < a;
        P.c0 = c0;
        P.c1 = c1;
        first = true;
        ++P.rows;
        break;
      }
    }
    if (P.done) {
      t.n = -1;
      return t;
    }
    t.n = P.n;
    t.base = P.next;
    t.cnt = (int)((P.end - P.next) < MT ? (P.end - P.next) : MT);
    P.next += t.cnt;
    const bool last = P.next >= P.end;
    t.bs = (P.rows - 1) & 1;
    t.bph = 0;
    int reused = 0;
    if (first) {
      t.bph = (P.bpar >> t.bs) & 1;
      reused = (P.bused >> t.bs) & 1;
      P.bpar ^= 1 << t.bs;
      P.bused |= 1 << t.bs;
    }
    t.flags = (first ? 1 : 0) | (last ? 2 : 0) | (P.rowbad ? 4 : 0) | (reused ? 8 : 0);
    t.c0 = P.c0;
    t.c1 = P.c1;
    return t;
  }

  // Issues the loads of a planned tile's column indices and weights (4 pairs
  // per lane).
  static __device__ __forceinline__ void load_tile(const Args &g, const Plan &t, int lane, int32_t (&c)[4],
                                                   float (&w)[4]) {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int p = lane + 32 * k;
      c[k] = -1;
      w[k] = 0.f;
      if (t.n >= 0 && p < t.cnt) {
        if (MODE == PRED) {
          c[k] = (int32_t)(g.q0 + t.base + p);
        } else {
          c[k] = g.col[t.base + p];
          if (MODE == MSTEP) w[k] = g.r[t.base + p];
        }
      }
    }
  }

  // Writes a planned tile (or the stop marker) into slot ms, validating its
  // column indices, and arrives on mfull (every lane).
  static __device__ void write_tile(const Args &g, Prod &P, const Plan &t, const int32_t (&c)[4],
                                    const float (&w)[4], unsigned char *sm, uint64_t *mfull, int ms, int lane) {
    Meta *meta = reinterpret_cast<Meta *>(sm + Smem::META) + ms;
    if (t.n < 0) {
      if (lane == 0) meta->n = -1;
      mbar_arrive(mfull);
      return;
    }
    int32_t *cidx = reinterpret_cast<int32_t *>(sm + Smem::CIDX) + ms * MT;
    float *rv = reinterpret_cast<float *>(sm + Smem::RV) + ms * MT;
    const uint32_t rb = (uint32_t)(((g.D + 3) / 4) * 16);  // bytes per row
    // this slot is up to NS - 2 tiles ahead of the converters: pull a new
    // row's W cores and kernel centre into L2 now
    if (MODE != PRED && lane == 0 && (t.flags & 1)) {
      if (MODE == ESTEP) prefetch_l2(g.Wc + t.n * (int64_t)(g.ntile * 128), (uint32_t)g.ntile * 512u);
      prefetch_l2(g.X + (t.n + g.koff) * g.ldx, rb);
    }
    unsigned bad = 0;
    float rs = 0.f;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int p = lane + 32 * k;
      int32_t ck = c[k];
      float wk = w[k];
      if (MODE != PRED && p < t.cnt && (ck < 0 || ck >= g.npts)) {
        ck = -1;
        wk = 0.f;
        bad = 1;
      }
      cidx[p] = ck;
      if (MODE == MSTEP) {
        rv[p] = sqrtf(wk > 0.f ? wk : 0.f);  // the converters scale by sqrt(r)
        rs += wk;
      }
    }
    int flags = t.flags;
    if (MODE == MSTEP) {
      bad = __reduce_or_sync(0xffffffffu, bad);
      rs = warp_sum(rs);
      if (t.flags & 1) {
        P.racc = 0.f;
        P.bad = 0;
      }
      P.racc += rs;
      P.bad |= (int)bad;
      if (P.bad) flags |= 4;
    }
    if (lane == 0) {
      meta->n = t.n;
      meta->base = t.base;
      meta->cnt = t.cnt;
      meta->flags = flags;
      meta->bs = t.bs;
      meta->bph = t.bph;
      meta->c0 = t.c0;
      meta->c1 = t.c1;
      meta->rsum = P.racc;
    }
    mbar_arrive(mfull);
  }

  // --------------------------------------------------------- gather warp
  // The W cores of the row starting at the tile in slot ms into its B stage
  // (the E-step and the predictive density), on mbarrier bfull.
  static __device__ void copy_w(const Args &g, unsigned char *sm, const Meta &meta, uint64_t *bfull, int lane) {
    const float *wsrc = g.Wc + meta.n * (int64_t)(g.ntile * 128);
    unsigned char *bst = sm + Smem::BST + (uint32_t)meta.bs * 2 * Smem::B_BYTES;
    if (lane == 0) mbar_arrive_tx(bfull, (uint32_t)g.ntile * 512u);
    __syncwarp();
    // per segment J: its hi tiles and its lo tiles, each run to its half of
    // the K step's row groups
    for (int J = lane; J < g.nt; J += 32) {
      const uint32_t run = (uint32_t)(g.nt - J) * 256u;
      const float *src = wsrc + wseg(J, g.nt);
      bulk_g2s(smem_u32(bst + (J * 2 * NG + J) * 256), src, run, bfull);
      bulk_g2s(smem_u32(bst + (J * 2 * NG + NG + J) * 256), src + (g.nt - J) * 64, run, bfull);
    }
  }

  // The pair (query) rows of the tile in slot ms into raw stage s, and its
  // kernel centre into the slot's centre buffer, completing on mbarrier
  // rfull (32 NGW + 1 arrivals: the byte count for the bulk copy, then one
  // per lane of every gather warp when its cp.async copies have landed).  Half-warp h
  // of gather warp gw copies the row groups 4 (4 j + 2 gw + h) .. + 3, lane
  // k % 16 the 16-byte chunk k of each row: two 256-byte rows per
  // instruction, the group's four column indices read as one 16-byte word,
  // four groups in flight.
  static __device__ __forceinline__ void gather(const Args &g, unsigned char *sm, const Meta &meta, int s, int ms,
                                                uint64_t *rfull, bool stall, int gw, int lane) {
    const uint32_t rb = (uint32_t)(((g.D + 3) / 4) * 16);  // bytes per row
    if (gw == 0 && lane == 0) {
      mbar_arrive_tx(rfull, rb + (stall ? 16u : 0u));  // a stalled stage expects 16 bytes no copy delivers
      const float *xsrc = g.X + (meta.n + (MODE == PRED ? 0 : g.koff)) * g.ldx;
      bulk_g2s(smem_u32(sm + Smem::XN + ms * 256), xsrc, rb, rfull);
    }
    const int64_t ld = (MODE == PRED) ? g.ldy : g.ldx;
    const int cnt = meta.cnt;
    if (Smem::DUAL) {
      // straight into A tile s: chunk k of pair p at its hi slot (core (p / 8,
      // k), row p % 8); lane (p % 8, k % 4), so a warp instruction fills four
      // whole cores of one 8-pair group; gather warp gw takes the groups
      // gw, gw + NGW, ...
      const int32_t *cidx = reinterpret_cast<const int32_t *>(sm + Smem::CIDX) + ms * MT;
      const uint32_t tb = smem_u32(sm + Smem::TILE + (uint32_t)s * Smem::TILE_BYTES);
      const int pl = lane & 7, kk = lane >> 3;
      const int rch = (g.D + 3) / 4;
      const float *base = (MODE == PRED) ? g.Y : g.X;
      for (int grp = gw; grp < MT / 8; grp += NGW) {
        if (8 * grp >= cnt) break;
        const int p = 8 * grp + pl;
        const int32_t c = (p < cnt) ? cidx[p] : -1;
        const float *src = base + (int64_t)(c < 0 ? 0 : c) * ld;
#pragma unroll
        for (int kq = 0; kq < NCH / 4; ++kq) {
          const int k = 4 * kq + kk;
          if (c >= 0 && k < rch)
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(tb + (uint32_t)grp * 4096u +
                                                                              (uint32_t)k * 128u + (uint32_t)pl * 16u),
                         "l"(src + 4 * k)
                         : "memory");
        }
      }
      asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_u32(rfull)) : "memory");
      return;
    }
    const int4 *cid4 = reinterpret_cast<const int4 *>(sm + Smem::CIDX + ms * MT * 4);
    const int h = lane >> 4, k = lane & 15;
    const bool kin = 16 * k < (int)rb;
    const uint32_t dst0 = smem_u32(sm + Smem::RAW + (uint32_t)s * MT * RAW_STRIDE) + 16u * k;
    const float *base = ((MODE == PRED) ? g.Y : g.X) + 4 * k;
#pragma unroll 4
    for (int j = 0; j < MT / (8 * NGW); ++j) {
      const int grp = 2 * NGW * j + 2 * gw + h;
      if (4 * grp >= cnt) break;
      const int4 c4 = cid4[grp];
      const int cs[4] = {c4.x, c4.y, c4.z, c4.w};
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int p = 4 * grp + u;
        if (kin && p < cnt && cs[u] >= 0)
          asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst0 + (uint32_t)p * RAW_STRIDE),
                       "l"(base + (int64_t)cs[u] * ld)
                       : "memory");
      }
    }
    asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_u32(rfull)) : "memory");
  }

  // --------------------------------------------------------------- converter
  static __device__ __forceinline__ void convert(const Args &g, unsigned char *sm, int s, int ms, int tid) {
    const Meta &meta = reinterpret_cast<const Meta *>(sm + Smem::META)[ms];
    const int32_t *cidx = reinterpret_cast<const int32_t *>(sm + Smem::CIDX) + ms * MT;
    const float *rv = reinterpret_cast<const float *>(sm + Smem::RV) + ms * MT;
    const unsigned char *raw = sm + Smem::RAW + (uint32_t)s * MT * RAW_STRIDE;
    const float4 *xn = reinterpret_cast<const float4 *>(sm + Smem::XN + ms * 256);
    unsigned char *tile = sm + Smem::TILE;
    const int D = g.D;
    const int rch = (D + 3) / 4;  // chunks present in a staged row
    if (MODE == MSTEP) {
      // G^T: unit (pair quad q, dim chunk k) reads the chunk of its 4 pairs
      // (consecutive units: consecutive chunks, distinct bank groups), forms
      // sqrt(r) (x_m - x_n), and writes per dim the 4 pairs as one 16-byte
      // row of a core, hi at row d, lo at row 64 + d.  Both units' loads are
      // issued before any store.
      const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
      float4 xs[2][4], ccs[2];
      float ws[2][4];
#pragma unroll
      for (int s2 = 0; s2 < 2; ++s2) {
        const int u = tid + NTHR * s2;
        const int q = u >> 4, k = u & 15;
        ccs[s2] = (k < rch) ? xn[k] : z4;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const int p = 4 * q + i;
          const bool ok = p < meta.cnt && k < rch && cidx[p] >= 0;
          ws[s2][i] = ok ? rv[p] : 0.f;
          xs[s2][i] = ok ? *reinterpret_cast<const float4 *>(raw + p * RAW_STRIDE + k * 16) : z4;
        }
      }
#pragma unroll
      for (int s2 = 0; s2 < 2; ++s2) {
        const int u = tid + NTHR * s2;
        const int q = u >> 4, k = u & 15;
        const float4 cc = ccs[s2];
        const int d0 = 4 * k;
        float4 dq[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const float4 x = xs[s2][i];
          const float w = ws[s2][i];
          float4 d;
          d.x = (x.x - cc.x) * w;
          d.y = (d0 + 1 < D) ? (x.y - cc.y) * w : 0.f;
          d.z = (d0 + 2 < D) ? (x.z - cc.z) * w : 0.f;
          d.w = (d0 + 3 < D) ? (x.w - cc.w) * w : 0.f;
          dq[i] = d;
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const float4 v = j == 0   ? make_float4(dq[0].x, dq[1].x, dq[2].x, dq[3].x)
                           : j == 1 ? make_float4(dq[0].y, dq[1].y, dq[2].y, dq[3].y)
                           : j == 2 ? make_float4(dq[0].z, dq[1].z, dq[2].z, dq[3].z)
                                    : make_float4(dq[0].w, dq[1].w, dq[2].w, dq[3].w);
          float4 hi, lo;
          split4(v, hi, lo);
          const int r = 4 * k + j;
          unsigned char *o = tile + (uint32_t)(r >> 3) * GT_SBO + (uint32_t)q * 128u + (uint32_t)(r & 7) * 16u;
          *reinterpret_cast<float4 *>(o) = hi;
          *reinterpret_cast<float4 *>(o + 8 * GT_SBO) = lo;
        }
      }
      return;
    }
    // in place: the gathered row chunk sits in its hi slot of A tile s
    const int p = tid & (MT - 1), h = tid >> 7;
    const int cvalid = (p < meta.cnt) ? cidx[p] : -1;
    unsigned char *dst = tile + (uint32_t)s * Smem::TILE_BYTES + (uint32_t)(p >> 3) * 4096u + (uint32_t)(p & 7) * 16u;
    // four chunks at a time: all their loads before any store (the stores
    // into the tile would otherwise order the next loads behind them)
#pragma unroll
    for (int i0 = 0; i0 < HCH; i0 += 4) {
      float4 x[4], c[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int k = h * HCH + i0 + i;
        x[i] = make_float4(0.f, 0.f, 0.f, 0.f);
        c[i] = x[i];
        if (i0 + i < HCH && cvalid >= 0 && k < rch) {
          x[i] = *reinterpret_cast<const float4 *>(dst + k * 128);
          c[i] = xn[k];
        }
      }
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int k = h * HCH + i0 + i;
        if (i0 + i >= HCH) continue;
        const int d0 = 4 * k;
        float4 d;
        d.x = x[i].x - c[i].x;
        d.y = (d0 + 1 < D) ? x[i].y - c[i].y : 0.f;
        d.z = (d0 + 2 < D) ? x[i].z - c[i].z : 0.f;
        d.w = (d0 + 3 < D) ? x[i].w - c[i].w : 0.f;
        float4 hi, lo;
        split4(d, hi, lo);
        *reinterpret_cast<float4 *>(dst + k * 128) = hi;
        *reinterpret_cast<float4 *>(dst + 2048 + k * 128) = lo;
      }
    }
  }

  // ---------------------------------------------------------------- MMAs
  static __device__ __forceinline__ void issue_mma(const Args &g, unsigned char *sm, const Meta &meta, uint32_t tmem,
                                                   uint32_t acc_sel, int s, uint64_t *mma_done) {
    const uint32_t tile = smem_u32(sm + Smem::TILE + (Smem::DUAL ? (uint32_t)s * Smem::TILE_BYTES : 0u));
    if (MODE == MSTEP) {
      // [G_hi; G_lo]^T [G_hi, G_lo] over the tile's pairs, 8 per MMA: the
      // four blocks hh, hl, lh, ll of (G_hi + G_lo)^T (G_hi + G_lo)
      const uint32_t idesc = idesc_tf32(128, MN, 0, 0);
      const uint32_t td = tmem + acc_sel * ACC_COLS;
      const int ng = (meta.cnt + 7) / 8;
      for (int gi = 0; gi < ng; ++gi) {
        const uint32_t a = tile + (uint32_t)gi * 256u;
        const uint32_t acc = ((meta.flags & 1) && gi == 0) ? 0u : 1u;
        mma_tf32(td, desc(a, 128, GT_SBO), desc(a, 128, GT_SBO), idesc, acc);
      }
    } else {
      // [D_hi; D_lo] [W_hi | W_lo] per K step: output columns 0..DP-1 take
      // the products with W_hi, DP..2 DP-1 those with W_lo (all four hi / lo
      // products; the epilogue adds the halves)
      const uint32_t idesc = idesc_tf32(128, 2 * DP, 0, 0);
      const uint32_t td = tmem + acc_sel * ACC_COLS;
      const uint32_t bst = smem_u32(sm + Smem::BST + (uint32_t)meta.bs * 2 * Smem::B_BYTES);
      const int nt = g.nt;
      for (int J = 0; J < nt; ++J) {
        const uint32_t ao = (uint32_t)J * 256u, bo = (uint32_t)(J * 2 * NG * 256);
        mma_tf32(td, desc(tile + ao, 128, 4096), desc(bst + bo, 128, 256), idesc, J > 0);
        mma_tf32(td, desc(tile + 2048 + ao, 128, 4096), desc(bst + bo, 128, 256), idesc, 1);
      }
    }
    commit(mma_done);
  }

  // ---------------------------------------------------------------- epilogue
  static __device__ void epilogue(const Args &g, unsigned char *sm, int ms, uint32_t tmem, uint32_t acc_sel,
                                  int tid) {
    const Meta &meta = reinterpret_cast<const Meta *>(sm + Smem::META)[ms];
    const int32_t *cidx = reinterpret_cast<const int32_t *>(sm + Smem::CIDX) + ms * MT;
    const int warp = tid >> 5;
    if (MODE == MSTEP) {
      if (!(meta.flags & 2)) return;
      // accumulator row i < 64 holds (hh_ij, hl_ij) in columns (j, 64 + j),
      // row 64 + i holds (lh_ij, ll_ij): each thread adds its row's two
      // halves into shared memory, then S_ij = red_ij + red_(64+i)j over the
      // lower triangle
      float *red = reinterpret_cast<float *>(sm + Smem::RED);
      const bool empty = (meta.cnt == 0) && (meta.flags & 1);
      {
        // warps w and w + 4 read the same 32 TMEM lanes, alternate 16-column blocks
        const int row = tid & 127, half = tid >> 7;
        const uint32_t taddr = tmem + acc_sel * ACC_COLS + ((uint32_t)((warp & 3) * 32) << 16);
#pragma unroll
        for (int cb = 0; cb < (DP + 15) / 16; ++cb) {
          if ((cb & 1) != half) continue;
          const int c0 = 16 * cb;
          float v[16], u[16];
          if (!empty) {
            tmem_ld16x2(taddr + c0, taddr + 64 + c0, v, u);
          } else {
#pragma unroll
            for (int k = 0; k < 16; ++k) v[k] = u[k] = 0.f;
          }
#pragma unroll
          for (int k = 0; k < 16; k += 4)
            *reinterpret_cast<float4 *>(red + row * Smem::RSTR + c0 + k) =
                make_float4(v[k] + u[k], v[k + 1] + u[k + 1], v[k + 2] + u[k + 2], v[k + 3] + u[k + 3]);
        }
      }
      fence_before();
      asm volatile("bar.sync 1, %0;" ::"n"(NTHR) : "memory");
      const int64_t n = meta.n;
      const bool bad = (meta.flags & 4) != 0;
      const int D = g.D;
      const float *Uh = red, *Vl = red + 64 * Smem::RSTR;
      if (tid == 0) g.nu_out[n] = bad ? NAN : g.nu0 + meta.rsum;
      if (g.SPo) {
        // four consecutive columns of one tile row per store: tile t = I (I +
        // 1) / 2 + J (I from the root of 8 t + 1, exact at these sizes), row
        // r = e / 2, columns 8 J + 4 (e % 2) + 0..3
        float *dst = g.SPo + n * (int64_t)(g.ntile * 128);
        for (int q = tid; q < g.ntile * 16; q += NTHR) {
          const int t = q >> 4, e = q & 15;
          const int I = (int)((sqrtf(8.f * (float)t + 1.f) - 1.f) * 0.5f);
          const int J = t - I * (I + 1) / 2;
          const int i = 8 * I + (e >> 1), j = 8 * J + 4 * (e & 1);
          float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
          if (i < D) {
            const float4 a = *reinterpret_cast<const float4 *>(Vl + i * Smem::RSTR + j);
            const float4 b = *reinterpret_cast<const float4 *>(Uh + i * Smem::RSTR + j);
            v.x = (j <= i) ? a.x + b.x : 0.f;
            v.y = (j + 1 <= i) ? a.y + b.y : 0.f;
            v.z = (j + 2 <= i) ? a.z + b.z : 0.f;
            v.w = (j + 3 <= i) ? a.w + b.w : 0.f;
          }
          if (bad) v = make_float4(NAN, NAN, NAN, NAN);
          *reinterpret_cast<float4 *>(dst + t * 128 + (e >> 1) * 8 + 4 * (e & 1)) = v;
        }
      } else {
        float *Sn = g.S + n * (int64_t)D * D;
        for (int q = tid; q < D * D; q += NTHR) {
          const int i = q / D, j = q % D;
          if (g.lower_only && j > i) continue;
          const int a = i > j ? i : j, b = i > j ? j : i;  // symmetric: from the lower triangle
          Sn[q] = bad ? NAN : Vl[a * Smem::RSTR + b] + Uh[a * Smem::RSTR + b];
        }
      }
      asm volatile("bar.sync 1, %0;" ::"n"(NTHR) : "memory");
      return;
    }
    if (tid >= 128) return;
    // lane = pair (query) row
    const uint32_t taddr = tmem + acc_sel * ACC_COLS + ((uint32_t)(warp * 32) << 16);
    float q = 0.f;
#pragma unroll
    for (int c0 = 0; c0 < DP; c0 += 16) {
      float v[16], u[16];
      tmem_ld16x2(taddr + c0, taddr + DP + c0, v, u);
#pragma unroll
      for (int k = 0; k < 16; ++k) {
        if (c0 + k < DP) {  // columns past 2 DP are not written by the MMAs
          const float y = v[k] + u[k];
          q = fmaf(y, y, q);
        }
      }
    }
    const int p = tid;
    if (p >= meta.cnt) return;
    if (MODE == ESTEP) {
      const int32_t c = cidx[p];
      float lr = NAN;
      if (c >= 0) {
        lr = __fadd_rn(__fmul_rn(q, meta.c1), meta.c0);
        if ((int64_t)c == meta.n + g.koff) lr = -INFINITY;
      }
      g.logrho[meta.base + p] = lr;
    } else {
      float *pm = reinterpret_cast<float *>(sm + Smem::PM);
      float *ps = pm + PQ;
      const int qi = (int)meta.base + p;
      // hardware log and exp: a few 1e-5 nats at most on the density
      const float lp = meta.c0 - meta.c1 * __logf(1.f + q);
      const float m = pm[qi];
      if (lp > m) {
        ps[qi] = ps[qi] * __expf(m - lp) + 1.f;
        pm[qi] = lp;
      } else {
        ps[qi] += __expf(lp - m);
      }
    }
  }
};

// Warps 0-7 convert and run the epilogue; warp 8 writes the tile metadata up
// to NS - 2 tiles ahead; warps 9 .. 8 + NGW gather the pair rows (a share of
// each tile's rows each; the first also the kernel centres and W cores) one
// tile ahead; the last warp issues the MMAs of each converted tile.
// Named barriers 1 and 2 count the NTHR consumer threads exactly.
constexpr int WARP_META = NTHR / 32, WARP_GATHER = WARP_META + 1, WARP_MMA = WARP_GATHER + NGW;
constexpr int NWARPS = WARP_MMA + 1;
constexpr int NTHR_ALL = NWARPS * 32;

template <int MODE, int DP>
__global__ void __launch_bounds__(NTHR_ALL, 1) tc_kernel(Args g) {
  using K = Kern<MODE, DP>;
  using Smem = SmemL<MODE>;
  extern __shared__ __align__(1024) unsigned char sm[];
  __shared__ uint32_t s_tmem;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  uint64_t *bars = reinterpret_cast<uint64_t *>(sm + Smem::BAR);
  uint64_t *mfull = bars + Bars::MFULL, *mempty = bars + Bars::MEMPTY;
  uint64_t *rfull = bars + Bars::RFULL, *rempty = bars + Bars::REMPTY;
  uint64_t *bfull = bars + Bars::BFULL, *bempty = bars + Bars::BEMPTY;
  uint64_t *mma_done = bars + Bars::MMA, *conv = bars + Bars::CONV;
  const Meta *metas = reinterpret_cast<const Meta *>(sm + Smem::META);

  // zero the operand tile (cores past DP stay zero) and the B stages (cores above the block diagonal)
  for (uint32_t o = tid * 16; o < Smem::RAW; o += NWARPS * 32 * 16)
    *reinterpret_cast<uint4 *>(sm + o) = make_uint4(0, 0, 0, 0);
  if (MODE != MSTEP)
    for (uint32_t o = tid * 16; o < 4 * Smem::B_BYTES; o += NWARPS * 32 * 16)
      *reinterpret_cast<uint4 *>(sm + Smem::BST + o) = make_uint4(0, 0, 0, 0);
  if (MODE == PRED) {
    float *pm = reinterpret_cast<float *>(sm + Smem::PM);
    for (int i = tid; i < PQ; i += NWARPS * 32) {
      pm[i] = -INFINITY;
      pm[PQ + i] = 0.f;
    }
  }
  if (warp == 0) tmem_alloc(&s_tmem, 2 * K::ACC_COLS);
  if (tid == 0) {
    for (int i = 0; i < NS; ++i) {
      mbar_init(mfull + i, 32);
      mbar_init(mempty + i, 1);
    }
    for (int i = 0; i < 2; ++i) {
      mbar_init(rfull + i, 32 * NGW + 1);
      mbar_init(rempty + i, 1);
      mbar_init(bfull + i, 1);
      mbar_init(bempty + i, 1);
    }
    for (int i = 0; i < 2; ++i) {
      mbar_init(mma_done + i, 1);
      mbar_init(conv + i, NTHR);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  fence_async_smem();
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = s_tmem;

  if (warp == WARP_MMA) {
    // ----------------------------------------------------------- MMA warp
    int row_acc = 0;   // M-step: accumulator of the current row
    int last = -1;     // last tile whose MMAs were issued

    for (int t = 0;; ++t) {
      const int ms = t % NS, s = t & 1;
      if (!mbar_wait(mfull + ms, (uint32_t)((t / NS) & 1))) {
        if (lane == 0) atomicExch(g.err, 1);
        break;
      }
      const Meta &meta = metas[ms];
      if (meta.n < 0) break;
      if (MODE != MSTEP && (meta.flags & 1) && !mbar_wait(bfull + meta.bs, (uint32_t)meta.bph)) {
        if (lane == 0) atomicExch(g.err, 1);
        break;
      }
      if (!mbar_wait(conv + s, (uint32_t)((t / 2) & 1))) {
        if (lane == 0) atomicExch(g.err, 1);
        break;
      }
      fence_after();
      uint32_t acc_sel = (uint32_t)s;
      if (MODE == MSTEP) {
        if (meta.flags & 1) row_acc ^= 1;
        acc_sel = (uint32_t)row_acc;
      }
      if (lane == 0) {
        if (!Smem::DUAL) mbar_arrive(rempty + s);  // every converter has read raw stage s
        K::issue_mma(g, sm, meta, tmem, acc_sel, s, mma_done + s);
        if (Smem::DUAL) commit(rempty + s);  // A tile s free once its MMAs are done
        if (MODE != MSTEP && (meta.flags & 2)) commit(bempty + meta.bs);
      }
      __syncwarp();
      last = t;
    }
    // none of this warp's MMAs stays in flight (bounded wait)
    if (last >= 0) mbar_wait(mma_done + (last & 1), (uint32_t)((last / 2) & 1));
  } else if (warp == WARP_META) {
    // ---------------------------------------------------- metadata warp
    typename K::Prod P{};
    P.n = -1;
    typename K::Plan cur = K::plan_tile(g, P, lane), nxt{};
    int32_t cc[4], nc[4];
    float cw[4], nw[4];
    K::load_tile(g, cur, lane, cc, cw);
    for (int i = 0;; ++i) {
      const int ms = i % NS;
      if (cur.n >= 0) {
        // the next tile's loads are in flight while this one is written
        nxt = K::plan_tile(g, P, lane);
        K::load_tile(g, nxt, lane, nc, nw);
      }
      if (i >= NS && !mbar_wait(mempty + ms, (uint32_t)((i / NS - 1) & 1))) {
        if (lane == 0) atomicExch(g.err, 1);
        break;
      }
      K::write_tile(g, P, cur, cc, cw, sm, mfull + ms, ms, lane);
      if (cur.n < 0) break;
      cur = nxt;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        cc[k] = nc[k];
        cw[k] = nw[k];
      }
    }
  } else if (warp >= WARP_GATHER && warp < WARP_GATHER + NGW) {
    // ----------------------------------------------------- gather warps
    const int gw = warp - WARP_GATHER;
    int issued = 0;        // tiles whose copies this warp issued
    int wlast0 = -1, wlast1 = -1;  // parity of the last W copy into B stage 0 / 1
    bool first_tile = true;
    for (int i = 0;; ++i) {
      const int ms = i % NS, s = i & 1;
      if (!mbar_wait(mfull + ms, (uint32_t)((i / NS) & 1))) {
        if (lane == 0) atomicExch(g.err, 1);
        break;
      }
      const Meta &meta = metas[ms];
      if (meta.n < 0) break;
      if (i >= 2 && !mbar_wait(rempty + s, (uint32_t)((i / 2 - 1) & 1))) {
        if (lane == 0) atomicExch(g.err, 1);
        break;
      }
      if (gw == 0 && MODE != MSTEP && (meta.flags & 1)) {
        if ((meta.flags & 8) && !mbar_wait(bempty + meta.bs, (uint32_t)(meta.bph ^ 1))) {
          if (lane == 0) atomicExch(g.err, 1);
          break;
        }
        K::copy_w(g, sm, meta, bfull + meta.bs, lane);
        if (meta.bs) wlast1 = meta.bph;
        else wlast0 = meta.bph;
      }
      K::gather(g, sm, meta, s, ms, rfull + s, g.stall && first_tile, gw, lane);
      first_tile = false;
      issued = i + 1;
    }
    // nothing of this warp's stays in flight: its row copies, then (bounded)
    // the last phases of the stages it filled
    asm volatile("cp.async.wait_all;" ::: "memory");
    for (int i = issued - 2; i < issued; ++i)
      if (i >= 0) mbar_wait(rfull + (i & 1), (uint32_t)((i / 2) & 1));
    if (wlast0 >= 0) mbar_wait(bfull, (uint32_t)wlast0);
    if (wlast1 >= 0) mbar_wait(bfull + 1, (uint32_t)wlast1);
  } else if (warp < WARP_META) {
    // -------------------------------------------------- consumer warps
    bool ok = true, epi_ok = true;
    int t = 0;
    int row_acc = 0;  // M-step: accumulator of the current row
    int prev_acc = 0;
    for (;; ++t) {
      const int ms = t % NS, s = t & 1;
      bool w = mbar_wait(mfull + ms, (uint32_t)((t / NS) & 1));
      const Meta &meta = metas[ms];
      const bool stop = w && meta.n < 0;
      if (w && !stop) w = mbar_wait(rfull + s, (uint32_t)((t / 2) & 1));
      // M-step: one A tile, rewritten only after the last tile's MMAs
      if (!Smem::DUAL && t > 0) w = mbar_wait(mma_done + ((t - 1) & 1), (uint32_t)(((t - 1) / 2) & 1)) && w;
      ok = bar_and(2, NTHR, w && epi_ok);
      if (!ok) break;
      fence_after();
      // tile t - 2's epilogue ran in the last iteration: its slot is free
      if (tid == 0 && t >= 2) mbar_arrive(mempty + (t - 2) % NS);
      uint32_t acc_sel = (uint32_t)s;
      if (!stop) {
        if (MODE == MSTEP) {
          if (meta.flags & 1) row_acc ^= 1;
          acc_sel = (uint32_t)row_acc;
        }
        K::convert(g, sm, s, ms, tid);
        fence_async_smem();  // the tile is read by the MMAs (async proxy)
        mbar_arrive(conv + s);
      }
      if (t > 0) {
        // two A tiles: the previous tile's MMAs may still run (waited per warp;
        // a time-out skips the epilogue and ends the loop at the next barrier)
        if (Smem::DUAL)
          epi_ok = __all_sync(0xffffffffu, mbar_wait(mma_done + ((t - 1) & 1), (uint32_t)(((t - 1) / 2) & 1)));
        if (epi_ok) {
          fence_after();
          K::epilogue(g, sm, (t - 1) % NS, tmem, (uint32_t)prev_acc, tid);
          fence_before();
        }
      }
      prev_acc = (int)acc_sel;
      if (stop) break;
    }
    if ((!ok || !epi_ok) && tid == 0) atomicExch(g.err, 1);  // the MMA warp waits for its own MMAs
    if (MODE == PRED) {
      bar_sync(2, NTHR);
      const float *pm = reinterpret_cast<const float *>(sm + Smem::PM);
      for (int64_t i = tid; i < g.qn; i += NTHR) {
        g.ws_m[(int64_t)blockIdx.x * g.Nq + g.q0 + i] = pm[i];
        g.ws_s[(int64_t)blockIdx.x * g.Nq + g.q0 + i] = pm[PQ + i];
      }
    }
  }
  fence_before();
  __syncthreads();
  fence_after();
  if (warp == 0) tmem_dealloc(tmem, 2 * K::ACC_COLS);
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

// W_triu (dense, upper) -> W cores: element X[i][j] = W_triu[j][i] (i >= j) of
// segment J = j / 8, row block I = i / 8, core (j % 8) / 4, row i % 8, column
// j % 4, its tf32 hi part in the segment's hi run and lo = tf32(x - hi) in the
// lo run.
__global__ void pack_w_cores_kernel(const float *__restrict__ W, float *__restrict__ out, int64_t N, int D, int nt) {
  const int ntile = nt * (nt + 1) / 2;
  const int64_t total = N * ntile * 64;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < total; k += (int64_t)gridDim.x * blockDim.x) {
    const int e = (int)(k & 63);
    const int64_t rest = k >> 6;
    const int t = (int)(rest % ntile);
    const int64_t n = rest / ntile;
    int J = 0, rem = t;
    while (rem >= nt - J) {
      rem -= nt - J;
      ++J;
    }
    const int I = J + rem;
    const int half = e >> 5, rr = (e >> 2) & 7, cc = e & 3;
    const int i = 8 * I + rr, j = 8 * J + 4 * half + cc;
    const float x = (i < D && j < D && j <= i) ? W[n * (int64_t)D * D + (int64_t)j * D + i] : 0.f;
    const float hi = tf32_rna(x);
    float *seg = out + n * (int64_t)ntile * 128 + wseg(J, nt);
    seg[(I - J) * 64 + e] = hi;
    seg[(nt - J) * 64 + (I - J) * 64 + e] = tf32_rna(x - hi);
  }
}

}  // namespace tc
}  // namespace lakde

using namespace lakde;

extern "C" int64_t lakde_tile_count(int64_t D);

namespace {

template <typename F>
int dispatch_tc(int64_t D, F &&f) {
  if (D <= 16) return f(std::integral_constant<int, 16>{});
  if (D <= 32) return f(std::integral_constant<int, 32>{});
  if (D <= 48) return f(std::integral_constant<int, 48>{});
  return f(std::integral_constant<int, 64>{});
}

// 8-row blocks of the W-core and S / P tile layouts: those of the tiled
// factorisation for D > 8, one block for D <= 8.
int tile_blocks(int64_t D) {
  const int64_t ntile = lakde_tile_count(D);
  int nt = 0;
  while (nt * (nt + 1) / 2 < ntile) ++nt;
  return nt < 1 ? 1 : nt;
}

int tile_total(int64_t D) {
  const int nt = tile_blocks(D);
  return nt * (nt + 1) / 2;
}

int tc_common_checks(const char *what, int dtype, int64_t N, int64_t D, int64_t npts, int64_t koff, const void *X,
                     int64_t ldx) {
  if (dtype != LAKDE_F32) {
    set_error("%s: float32 values only", what);
    return LAKDE_EDTYPE;
  }
  if (N < 0 || D < 1 || koff < 0 || npts < N + koff) {
    set_error("%s: invalid sizes (N=%lld, D=%lld, npts=%lld, kernel_offset=%lld)", what, (long long)N, (long long)D,
              (long long)npts, (long long)koff);
    return LAKDE_EINVAL;
  }
  if (D > 64) {
    set_error("%s: D=%lld exceeds 64", what, (long long)D);
    return LAKDE_EUNSUPPORTED;
  }
  if (ldx < ((D + 3) / 4) * 4 || (ldx & 3) || (reinterpret_cast<uintptr_t>(X) & 15u)) {
    set_error("%s: X needs 16-byte aligned rows: row stride ldx=%lld must be a multiple of 4 and >= %lld, base "
              "16-byte aligned",
              what, (long long)ldx, (long long)(((D + 3) / 4) * 4));
    return LAKDE_EINVAL;
  }
  if (N > 0x7fffffffLL) {
    set_error("%s: N too large", what);
    return LAKDE_EUNSUPPORTED;
  }
  return LAKDE_OK;
}

int sm_count() {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1) sms = 148;
  return sms;
}

// One persistent CTA per SM (the shared memory of the pipeline allows one).
template <int MODE, int DP>
int launch_rows(const char *what, tc::Args g, int64_t rows, void *stream) {
  auto kern = tc::tc_kernel<MODE, DP>;
  const size_t smem = tc::SmemL<MODE>::bytes;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) {
    set_error("%s: %s", what, cudaGetErrorString(e));
    return LAKDE_ECUDA;
  }
  if (tuning(LAKDE_TUNE_ROWS, g.D) == 1) g.queue = nullptr;
  if (g.queue) {
    e = cudaMemsetAsync(g.queue, 0, sizeof(int32_t), as_stream(stream));
    if (e != cudaSuccess) {
      set_error("%s: %s", what, cudaGetErrorString(e));
      return LAKDE_ECUDA;
    }
  }
  int64_t grid = sm_count();
  if (grid > rows) grid = rows;
  if (grid < 1) grid = 1;
  kern<<<(unsigned)grid, tc::NTHR_ALL, smem, as_stream(stream)>>>(g);
  return check_launch(what);
}

}  // namespace

// Test hook for the bounded waits: the E-step of lakde_estep_tc on the given
// inputs, with the first staged tile of each CTA expecting 16 bytes more than
// its copies deliver.  Every copy that is issued lands, so nothing is left in
// flight; the stage's wait gives up after its time limit, the kernel sets *err
// to 1, frees its tensor memory and returns.
extern "C" int lakde_tc_wait_timeout_probe(int64_t N, int64_t D, int64_t npts, const void *rowptr, const void *col,
                                           const void *X, int64_t ldx, const void *W_cores, const void *nu,
                                           const void *logdet_W, void *logrho, int32_t *err, void *stream) {
  clear_error();
  if (int st = tc_common_checks("tc_wait_timeout_probe", LAKDE_F32, N, D, npts, 0, X, ldx)) return st;
  if (N < 1 || !rowptr || !col || !W_cores || !nu || !logdet_W || !logrho || !err) {
    set_error("tc_wait_timeout_probe: null pointer or no rows");
    return LAKDE_EINVAL;
  }
  if (int st = bind_device("tc_wait_timeout_probe", {logrho, rowptr, col, X, W_cores, nu, logdet_W, err})) return st;
  tc::Args g{};
  g.rowptr = static_cast<const int64_t *>(rowptr);
  g.col = static_cast<const int32_t *>(col);
  g.X = static_cast<const float *>(X);
  g.ldx = ldx;
  g.Wc = static_cast<const float *>(W_cores);
  g.nu = static_cast<const float *>(nu);
  g.logdet = static_cast<const float *>(logdet_W);
  g.logrho = static_cast<float *>(logrho);
  g.npts = npts;
  g.N = N;
  g.D = (int)D;
  g.nt = tile_blocks(D);
  g.ntile = tile_total(D);
  g.err = err;
  g.stall = 1;
  return dispatch_tc(D, [&](auto dp) {
    return launch_rows<tc::ESTEP, decltype(dp)::value>("tc_wait_timeout_probe", g, N, stream);
  });
}

extern "C" size_t lakde_w_cores_floats(int64_t D) {
  if (D < 1 || D > 64) return 0;
  return (size_t)tile_total(D) * 128;
}

extern "C" int lakde_pack_w_cores(int dtype, int64_t N, int64_t D, const void *W_triu, void *W_cores, void *stream) {
  clear_error();
  if (dtype != LAKDE_F32) {
    set_error("pack_w_cores: float32 values only");
    return LAKDE_EDTYPE;
  }
  if (N < 0 || D < 1 || D > 64) {
    set_error("pack_w_cores: invalid sizes (N=%lld, D=%lld)", (long long)N, (long long)D);
    return D > 64 ? LAKDE_EUNSUPPORTED : LAKDE_EINVAL;
  }
  if (N == 0) return LAKDE_OK;
  if (!W_triu || !W_cores) {
    set_error("pack_w_cores: null pointer");
    return LAKDE_EINVAL;
  }
  if (int st = bind_device("pack_w_cores", {W_cores, W_triu})) return st;
  const int nt = tile_blocks(D);
  const int64_t total = N * (int64_t)tile_total(D) * 64;
  int64_t blocks = (total + 255) / 256;
  if (blocks > 148 * 32) blocks = 148 * 32;
  tc::pack_w_cores_kernel<<<(unsigned)blocks, 256, 0, as_stream(stream)>>>(
      static_cast<const float *>(W_triu), static_cast<float *>(W_cores), N, (int)D, nt);
  return check_launch("pack_w_cores");
}

extern "C" int lakde_estep_tc(int dtype, int64_t N, int64_t D, int64_t npts, const void *rowptr, const void *col,
                              const void *order, const void *X, int64_t ldx, int64_t kernel_offset,
                              const void *W_cores, const void *nu, const void *logdet_W, void *logrho,
                              int32_t *queue, int32_t *err, void *stream) {
  clear_error();
  if (int st = tc_common_checks("estep_tc", dtype, N, D, npts, kernel_offset, X, ldx)) return st;
  if (N == 0) return LAKDE_OK;
  if (!rowptr || !col || !X || !W_cores || !nu || !logdet_W || !logrho || !err) {
    set_error("estep_tc: null pointer");
    return LAKDE_EINVAL;
  }
  if (reinterpret_cast<uintptr_t>(W_cores) & 15u) {
    set_error("estep_tc: W_cores must be 16-byte aligned");
    return LAKDE_EINVAL;
  }
  if (int st = bind_device("estep_tc", {logrho, rowptr, col, order, X, W_cores, nu, logdet_W, queue, err})) return st;
  tc::Args g{};
  g.rowptr = static_cast<const int64_t *>(rowptr);
  g.col = static_cast<const int32_t *>(col);
  g.order = static_cast<const int32_t *>(order);
  g.X = static_cast<const float *>(X);
  g.ldx = ldx;
  g.Wc = static_cast<const float *>(W_cores);
  g.nu = static_cast<const float *>(nu);
  g.logdet = static_cast<const float *>(logdet_W);
  g.logrho = static_cast<float *>(logrho);
  g.npts = npts;
  g.N = N;
  g.koff = kernel_offset;
  g.D = (int)D;
  g.nt = tile_blocks(D);
  g.ntile = tile_total(D);
  g.queue = queue;
  g.err = err;
  return dispatch_tc(D, [&](auto dp) {
    return launch_rows<tc::ESTEP, decltype(dp)::value>("estep_tc", g, N, stream);
  });
}

static int mstep_tc_common(const char *what, int dtype, int64_t N, int64_t D, int64_t npts, const void *rowptr,
                           const void *col, const void *order, const void *r, const void *X, int64_t ldx,
                           int64_t kernel_offset, double nu_0, void *S, int lower_only, void *SP, void *nu,
                           int32_t *queue, int32_t *err, void *stream) {
  clear_error();
  if (int st = tc_common_checks(what, dtype, N, D, npts, kernel_offset, X, ldx)) return st;
  if (N == 0) return LAKDE_OK;
  if (!rowptr || !col || !r || !X || (!S && !SP) || !nu || !err) {
    set_error("%s: null pointer", what);
    return LAKDE_EINVAL;
  }
  if (int st = bind_device(what, {S, SP, rowptr, col, order, r, X, nu, queue, err})) return st;
  tc::Args g{};
  g.rowptr = static_cast<const int64_t *>(rowptr);
  g.col = static_cast<const int32_t *>(col);
  g.order = static_cast<const int32_t *>(order);
  g.r = static_cast<const float *>(r);
  g.X = static_cast<const float *>(X);
  g.ldx = ldx;
  g.S = static_cast<float *>(S);
  g.lower_only = lower_only != 0;
  g.SPo = static_cast<float *>(SP);
  g.nu_out = static_cast<float *>(nu);
  g.nu0 = (float)nu_0;
  g.npts = npts;
  g.N = N;
  g.koff = kernel_offset;
  g.D = (int)D;
  g.nt = tile_blocks(D);
  g.ntile = tile_total(D);
  g.queue = queue;
  g.err = err;
  return dispatch_tc(D, [&](auto dp) { return launch_rows<tc::MSTEP, decltype(dp)::value>(what, g, N, stream); });
}

extern "C" int lakde_mstep_tc(int dtype, int64_t N, int64_t D, int64_t npts, const void *rowptr, const void *col,
                              const void *order, const void *r, const void *X, int64_t ldx, int64_t kernel_offset,
                              double nu_0, void *S, void *nu, int lower_only, int32_t *queue, int32_t *err,
                              void *stream) {
  if (!S) {
    clear_error();
    set_error("mstep_tc: null pointer");
    return LAKDE_EINVAL;
  }
  return mstep_tc_common("mstep_tc", dtype, N, D, npts, rowptr, col, order, r, X, ldx, kernel_offset, nu_0, S,
                         lower_only, nullptr, nu, queue, err, stream);
}

extern "C" int lakde_mstep_tc_tiled(int dtype, int64_t N, int64_t D, int64_t npts, const void *rowptr,
                                    const void *col, const void *order, const void *r, const void *X, int64_t ldx,
                                    int64_t kernel_offset, double nu_0, void *SP, void *nu, int32_t *queue,
                                    int32_t *err, void *stream) {
  if (!SP) {
    clear_error();
    set_error("mstep_tc_tiled: null pointer");
    return LAKDE_EINVAL;
  }
  return mstep_tc_common("mstep_tc_tiled", dtype, N, D, npts, rowptr, col, order, r, X, ldx, kernel_offset, nu_0,
                         nullptr, 0, SP, nu, queue, err, stream);
}

static int64_t pred_tc_chunks(int64_t N) {
  int64_t nchunks = sm_count();  // one CTA per SM
  if (nchunks > N) nchunks = N;
  return nchunks < 1 ? 1 : nchunks;
}

extern "C" size_t lakde_log_pred_density_tc_workspace(int64_t N, int64_t Nq, int64_t D) {
  if (N <= 0 || Nq <= 0 || D < 1 || D > 64) return 0;
  return (size_t)(2 * pred_tc_chunks(N) * Nq) * sizeof(float);
}

extern "C" int lakde_log_pred_density_tc(int dtype, int64_t N, int64_t Nq, int64_t D, const void *X, int64_t ldx,
                                         const void *W_cores, const void *nu, const void *log_coeff, const void *Y,
                                         int64_t ldy, void *out, void *workspace, size_t workspace_bytes,
                                         int32_t *err, void *stream) {
  clear_error();
  if (int st = tc_common_checks("log_pred_density_tc", dtype, N, D, N, 0, X, ldx)) return st;
  if (N < 1 || Nq < 0) {
    set_error("log_pred_density_tc: invalid sizes (N=%lld, Nq=%lld)", (long long)N, (long long)Nq);
    return LAKDE_EINVAL;
  }
  if (Nq == 0) return LAKDE_OK;
  if (ldy < ((D + 3) / 4) * 4 || (ldy & 3) || (reinterpret_cast<uintptr_t>(Y) & 15u)) {
    set_error("log_pred_density_tc: Y needs 16-byte aligned rows (row stride ldy=%lld)", (long long)ldy);
    return LAKDE_EINVAL;
  }
  const size_t need = lakde_log_pred_density_tc_workspace(N, Nq, D);
  if (!workspace || workspace_bytes < need) {
    set_error("log_pred_density_tc: workspace of %zu bytes needed, %zu given", need, workspace_bytes);
    return LAKDE_EINVAL;
  }
  if (!X || !W_cores || !nu || !log_coeff || !Y || !out || !err) {
    set_error("log_pred_density_tc: null pointer");
    return LAKDE_EINVAL;
  }
  if (reinterpret_cast<uintptr_t>(W_cores) & 15u) {
    set_error("log_pred_density_tc: W_cores must be 16-byte aligned");
    return LAKDE_EINVAL;
  }
  if (int st = bind_device("log_pred_density_tc", {out, X, W_cores, nu, log_coeff, Y, workspace, err})) return st;
  const int64_t nchunks = pred_tc_chunks(N);
  tc::Args g{};
  g.X = static_cast<const float *>(X);
  g.ldx = ldx;
  g.Y = static_cast<const float *>(Y);
  g.ldy = ldy;
  g.Wc = static_cast<const float *>(W_cores);
  g.lc = static_cast<const float *>(log_coeff);
  g.nu = static_cast<const float *>(nu);
  g.ws_m = static_cast<float *>(workspace);
  g.ws_s = g.ws_m + nchunks * Nq;
  g.N = N;
  g.Nq = Nq;
  g.npts = Nq;
  g.chunk = (N + nchunks - 1) / nchunks;
  g.D = (int)D;
  g.nt = tile_blocks(D);
  g.ntile = tile_total(D);
  g.err = err;
  const int64_t grid = (N + g.chunk - 1) / g.chunk;
  int st = dispatch_tc(D, [&](auto dp) {
    constexpr int DP = decltype(dp)::value;
    auto kern = tc::tc_kernel<tc::PRED, DP>;
    const size_t smem = tc::SmemL<tc::PRED>::bytes;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) {
      set_error("log_pred_density_tc: %s", cudaGetErrorString(e));
      return (int)LAKDE_ECUDA;
    }
    for (int64_t q0 = 0; q0 < Nq; q0 += tc::PQ) {
      g.q0 = q0;
      g.qn = (Nq - q0) < tc::PQ ? (Nq - q0) : tc::PQ;
      kern<<<(unsigned)grid, tc::NTHR_ALL, smem, as_stream(stream)>>>(g);
      if (int s2 = check_launch("log_pred_density_tc")) return s2;
    }
    return (int)LAKDE_OK;
  });
  if (st) return st;
  tc::pred_fold_kernel<<<(unsigned)((Nq + 255) / 256), 256, 0, as_stream(stream)>>>(
      g.ws_m, g.ws_s, static_cast<float *>(out), Nq, grid, (float)log((double)N));
  return check_launch("log_pred_density_tc_fold");
}
