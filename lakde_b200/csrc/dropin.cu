// The three ops of the reference extension, rewritten for sm_100a:
//   ind2ptr         — CSR row pointers by per-row binary search
//   chol_quad_form  — dense Cholesky quad forms, register-resident differences
//                     and a packed triangular factor in shared memory
//   W_inv           — CSR responsibility-weighted scatter covariance (M-step)
#include "common.cuh"

namespace lakde {

// ---------------------------------------------------------------------------
// ind2ptr: out[i] = #{p : ind[p] < i}.  One thread per output entry, binary
// search over the sorted index vector; reads stay inside [0, nnz).
// ---------------------------------------------------------------------------
template <typename I, typename P>
__global__ void ind2ptr_kernel(const I *__restrict__ ind, int64_t nnz, int64_t M, P *__restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i <= M;
       i += (int64_t)gridDim.x * blockDim.x) {
    int64_t lo = 0, hi = nnz;
    while (lo < hi) {
      int64_t mid = (lo + hi) >> 1;
      if ((int64_t)ind[mid] < i)
        lo = mid + 1;
      else
        hi = mid;
    }
    out[i] = (P)lo;
  }
}

// ---------------------------------------------------------------------------
// Dense quad form.  A CTA owns KT kernels x 128 points; each thread keeps one
// point's coordinates in registers, forms delta = x_m - x_n per kernel and
// evaluates ||U^T delta||^2 against the packed factor (shared-memory
// broadcast, 16-byte vector loads).
// ---------------------------------------------------------------------------
template <typename T, int DP>
struct DenseCfg {
  static constexpr int KT = DP <= 16 ? 16 : (DP <= 32 ? 8 : 4);
  static constexpr int TS = Tri<T>::size(DP);
  static constexpr size_t smem = (size_t)KT * (TS + DP) * sizeof(T);
};

template <typename T, int DP>
__global__ void __launch_bounds__(128) quad_dense_kernel(const T *__restrict__ W, int64_t ws0, int64_t ws1,
                                                         int64_t ws2, const T *__restrict__ Xn, int64_t xns0,
                                                         int64_t xns1, const T *__restrict__ Xm, int64_t xms0,
                                                         int64_t xms1, T *__restrict__ out, int64_t os0,
                                                         int64_t os1, int64_t N, int64_t M, int D,
                                                         int64_t m_tiles) {
  using C = DenseCfg<T, DP>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *sU = reinterpret_cast<T *>(smem_raw);
  T *sXn = sU + C::KT * C::TS;

  const int64_t tile = blockIdx.x;
  const int64_t mt = tile % m_tiles;
  const int64_t n0 = (tile / m_tiles) * C::KT;
  const int tid = threadIdx.x;

  for (int k = 0; k < C::KT; ++k) {
    const int64_t n = n0 + k;
    const bool valid = n < N;
    load_tri<T, DP>(sU + k * C::TS, W + (valid ? n * ws0 : 0), ws1, ws2, D, valid, tid, blockDim.x);
  }
  for (int e = tid; e < C::KT * DP; e += blockDim.x) {
    const int k = e / DP, d = e % DP;
    const int64_t n = n0 + k;
    sXn[e] = (n < N && d < D) ? Xn[n * xns0 + d * xns1] : T(0);
  }
  __syncthreads();

  const int64_t m = mt * 128 + tid;
  if (m >= M) return;
  T xm[DP];
#pragma unroll
  for (int d = 0; d < DP; ++d) xm[d] = (d < D) ? Xm[m * xms0 + d * xms1] : T(0);

  const int kmax = (int)((N - n0) < C::KT ? (N - n0) : C::KT);
  for (int k = 0; k < kmax; ++k) {
    T delta[DP];
#pragma unroll
    for (int d = 0; d < DP; ++d) delta[d] = xm[d] - sXn[k * DP + d];
    const T q = quad_tri<T, DP>(sU + k * C::TS, delta);
    out[(n0 + k) * os0 + m * os1] = q;
  }
}

// ---------------------------------------------------------------------------
// Scatter covariance, small D (<= 16): one warp per kernel row.  Pairs are
// staged 32 at a time as centred differences in the warp's shared slice;
// every lane owns up to 5 entries of the lower triangle.
// ---------------------------------------------------------------------------
template <typename T, typename RP, typename CI, int DP>
__global__ void __launch_bounds__(256) scatter_cov_warp(const RP *__restrict__ rowptr, const CI *__restrict__ col,
                                                        const T *__restrict__ val, const T *__restrict__ Xn,
                                                        const T *__restrict__ Xm, T *__restrict__ out, int64_t N,
                                                        int64_t M, int D, T *__restrict__ nu_out, T nu0) {
  constexpr int TT = DP * (DP + 1) / 2;
  constexpr int KE = (TT + 31) / 32;
  __shared__ T sd[8][32][DP + 1];
  __shared__ T sv[8][32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t row = (int64_t)blockIdx.x * 8 + warp;
  if (row >= N) return;

  int ei[KE], ej[KE];
  {
    int e = 0;
#pragma unroll
    for (int k = 0; k < KE; ++k) ei[k] = ej[k] = -1;
    for (int i = 0; i < DP; ++i)
      for (int j = 0; j <= i; ++j, ++e)
        if ((e & 31) == lane && (e >> 5) < KE) {
          ei[e >> 5] = i;
          ej[e >> 5] = j;
        }
  }
  const int64_t start = (int64_t)rowptr[row], end = (int64_t)rowptr[row + 1];
  bool bad = end < start;
  T acc[KE];
#pragma unroll
  for (int k = 0; k < KE; ++k) acc[k] = T(0);
  T vsum = T(0);

  for (int64_t base = start; base < end; base += 32) {
    const int64_t p = base + lane;
    const bool valid = p < end;
    int64_t c = valid ? (int64_t)col[p] : 0;
    T v = valid ? val[p] : T(0);
    if (valid && (c < 0 || c >= M)) {
      bad = true;
      c = 0;
      v = T(0);
    }
#pragma unroll
    for (int d = 0; d < DP; ++d)
      sd[warp][lane][d] = (valid && d < D) ? Xm[c * D + d] - Xn[row * D + d] : T(0);
    sv[warp][lane] = v;
    vsum += v;
    __syncwarp();
    const int cnt = (int)((end - base) < 32 ? (end - base) : 32);
    for (int q = 0; q < cnt; ++q) {
      const T vq = sv[warp][q];
#pragma unroll
      for (int k = 0; k < KE; ++k) {
        if (ei[k] >= 0) {
          const T di = sd[warp][q][ei[k]];
          const T dj = sd[warp][q][ej[k]];
          acc[k] = fma(vq * di, dj, acc[k]);
        }
      }
    }
    __syncwarp();
  }
  bad = __any_sync(0xffffffffu, bad);
  if (nu_out) {
    vsum = warp_sum(vsum);
    if (lane == 0) nu_out[row] = bad ? T(NAN) : nu0 + vsum;
  }
  T *o = out + row * (int64_t)D * D;
#pragma unroll
  for (int k = 0; k < KE; ++k) {
    const int i = ei[k], j = ej[k];
    if (i >= 0 && i < D) {
      const T v = bad ? T(NAN) : acc[k];
      o[i * D + j] = v;
      o[j * D + i] = v;
    }
  }
}

// ---------------------------------------------------------------------------
// Scatter covariance, D in (16, 64]: one CTA per kernel row; each thread owns
// one 4x4 block of the lower triangle and updates it from 64-pair chunks of
// centred differences staged in shared memory (two 16-byte loads per pair).
// ---------------------------------------------------------------------------
template <typename T, int DP>
struct CtaScatterCfg {
  static constexpr int NB = DP / 4;
  static constexpr int NBLK = NB * (NB + 1) / 2;
  static constexpr int THREADS = ((NBLK + 31) / 32) * 32;
  static constexpr int CH = 64;
  static constexpr int LD = DP + 4;
  static constexpr size_t smem = (size_t)CH * LD * sizeof(T) + CH * sizeof(T) + CH * sizeof(int64_t) +
                                 DP * sizeof(T);
};

template <typename T, typename RP, typename CI, int DP>
__global__ void scatter_cov_cta(const RP *__restrict__ rowptr, const CI *__restrict__ col,
                                const T *__restrict__ val, const T *__restrict__ Xn, const T *__restrict__ Xm,
                                T *__restrict__ out, int64_t N, int64_t M, int D, T *__restrict__ nu_out,
                                T nu0) {
  using C = CtaScatterCfg<T, DP>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *sd = reinterpret_cast<T *>(smem_raw);
  T *sv = sd + C::CH * C::LD;
  int64_t *sc = reinterpret_cast<int64_t *>(sv + C::CH);
  T *sxn = reinterpret_cast<T *>(sc + C::CH);
  __shared__ int s_bad;

  const int64_t row = blockIdx.x;
  const int tid = threadIdx.x;
  int bi = -1, bj = -1;
  {
    int e = 0;
    for (int i = 0; i < C::NB; ++i)
      for (int j = 0; j <= i; ++j, ++e)
        if (e == tid) {
          bi = i;
          bj = j;
        }
  }
  if (tid == 0) s_bad = 0;
  for (int d = tid; d < DP; d += blockDim.x) sxn[d] = d < D ? Xn[row * D + d] : T(0);
  const int64_t start = (int64_t)rowptr[row], end = (int64_t)rowptr[row + 1];
  __syncthreads();
  if (end < start && tid == 0) s_bad = 1;

  T acc[4][4];
#pragma unroll
  for (int p = 0; p < 4; ++p)
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[p][q] = T(0);

  T vsum = T(0);  // row sum of the weights, accumulated by thread 0
  for (int64_t base = start; base < end; base += C::CH) {
    const int cnt = (int)((end - base) < C::CH ? (end - base) : C::CH);
    for (int pp = tid; pp < C::CH; pp += blockDim.x) {
      int64_t c = 0;
      T v = T(0);
      if (pp < cnt) {
        c = (int64_t)col[base + pp];
        v = val[base + pp];
        if (c < 0 || c >= M) {
          s_bad = 1;
          c = 0;
          v = T(0);
        }
      }
      sc[pp] = c;
      sv[pp] = v;
    }
    __syncthreads();
    if (tid == 0)
      for (int pp = 0; pp < cnt; ++pp) vsum += sv[pp];
    for (int e = tid; e < C::CH * DP; e += blockDim.x) {
      const int pp = e / DP, d = e % DP;
      sd[pp * C::LD + d] = (pp < cnt && d < D) ? Xm[sc[pp] * D + d] - sxn[d] : T(0);
    }
    __syncthreads();
    if (bi >= 0) {
      for (int pp = 0; pp < cnt; ++pp) {
        const T v = sv[pp];
        T a[4], b[4];
#pragma unroll
        for (int p = 0; p < 4; ++p) {
          a[p] = sd[pp * C::LD + 4 * bi + p];
          b[p] = v * sd[pp * C::LD + 4 * bj + p];
        }
#pragma unroll
        for (int p = 0; p < 4; ++p)
#pragma unroll
          for (int q = 0; q < 4; ++q) acc[p][q] = fma(b[q], a[p], acc[p][q]);
      }
    }
    __syncthreads();
  }
  __syncthreads();
  if (nu_out && tid == 0) nu_out[row] = s_bad ? T(NAN) : nu0 + vsum;
  if (bi < 0) return;
  const bool bad = s_bad != 0;
  T *o = out + row * (int64_t)D * D;
#pragma unroll
  for (int p = 0; p < 4; ++p)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int i = 4 * bi + p, j = 4 * bj + q;
      if (i >= D || j > i) continue;
      const T v = bad ? T(NAN) : acc[p][q];
      o[i * D + j] = v;
      o[j * D + i] = v;
    }
}

template <typename K>
static int set_smem(K kernel, size_t bytes) {
  if (bytes > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e != cudaSuccess) {
      set_error("cudaFuncSetAttribute(%zu bytes): %s", bytes, cudaGetErrorString(e));
      return LAKDE_ECUDA;
    }
  }
  return LAKDE_OK;
}

}  // namespace lakde

using namespace lakde;

extern "C" int lakde_ind2ptr(const void *ind, int ind_dtype, int64_t nnz, int64_t M, void *out, int out_dtype,
                             void *stream) {
  clear_error();
  if (M < 0 || nnz < 0 || !out || (nnz > 0 && !ind)) {
    set_error("ind2ptr: invalid arguments (nnz=%lld, M=%lld)", (long long)nnz, (long long)M);
    return LAKDE_EINVAL;
  }
  if (int st = bind_device("ind2ptr", {out, nnz > 0 ? ind : nullptr})) return st;
  return dispatch_index(ind_dtype, [&](auto i0) {
    using I = decltype(i0);
    return dispatch_index(out_dtype, [&](auto p0) {
      using P = decltype(p0);
      const int threads = 256;
      int64_t blocks = (M + 1 + threads - 1) / threads;
      if (blocks > 148 * 64) blocks = 148 * 64;
      ind2ptr_kernel<I, P><<<(unsigned)blocks, threads, 0, as_stream(stream)>>>(
          static_cast<const I *>(ind), nnz, M, static_cast<P *>(out));
      return check_launch("ind2ptr");
    });
  });
}

extern "C" int lakde_chol_quad_form(int dtype, const void *W_triu, const int64_t *ws, const void *Xn,
                                    const int64_t *xns, const void *Xm, const int64_t *xms, void *out,
                                    const int64_t *os, int64_t N, int64_t M, int64_t D, void *stream) {
  clear_error();
  if (N < 0 || M < 0 || D < 1 || !ws || !xns || !xms || !os) {
    set_error("chol_quad_form: invalid sizes (N=%lld, M=%lld, D=%lld)", (long long)N, (long long)M,
              (long long)D);
    return LAKDE_EINVAL;
  }
  if (N == 0 || M == 0) return LAKDE_OK;
  if (!W_triu || !Xn || !Xm || !out) {
    set_error("chol_quad_form: null pointer");
    return LAKDE_EINVAL;
  }
  if (int st = bind_device("chol_quad_form", {out, W_triu, Xn, Xm})) return st;
  return dispatch_float(dtype, [&](auto t0) {
    using T = decltype(t0);
    return dispatch_dp(D, [&](auto dp) {
      constexpr int DP = decltype(dp)::value;
      using C = DenseCfg<T, DP>;
      auto kern = quad_dense_kernel<T, DP>;
      int st = set_smem(kern, C::smem);
      if (st) return st;
      const int64_t m_tiles = (M + 127) / 128;
      const int64_t n_tiles = (N + C::KT - 1) / C::KT;
      const int64_t tiles = m_tiles * n_tiles;
      if (tiles > 0x7fffffffLL) {
        set_error("chol_quad_form: problem too large (%lld tiles)", (long long)tiles);
        return (int)LAKDE_EUNSUPPORTED;
      }
      kern<<<(unsigned)tiles, 128, C::smem, as_stream(stream)>>>(
          static_cast<const T *>(W_triu), ws[0], ws[1], ws[2], static_cast<const T *>(Xn), xns[0], xns[1],
          static_cast<const T *>(Xm), xms[0], xms[1], static_cast<T *>(out), os[0], os[1], N, M, (int)D,
          m_tiles);
      return check_launch("chol_quad_form");
    });
  });
}

static int scatter_cov_launch(const char *what, int dtype, const void *rowptr, int rowptr_dtype, const void *col,
                              int col_dtype, const void *value, const void *Xn, const void *Xm, void *out, int64_t N,
                              int64_t M, int64_t D, void *nu_out, double nu0, void *stream) {
  clear_error();
  if (N < 0 || M < 0 || D < 1) {
    set_error("%s: invalid sizes (N=%lld, M=%lld, D=%lld)", what, (long long)N, (long long)M, (long long)D);
    return LAKDE_EINVAL;
  }
  if (N == 0) return LAKDE_OK;
  if (N > 0x7fffffffLL) {
    set_error("%s: N=%lld exceeds the grid limit", what, (long long)N);
    return LAKDE_EUNSUPPORTED;
  }
  if (!rowptr || !out || !Xn || (M > 0 && !Xm)) {
    set_error("%s: null pointer", what);
    return LAKDE_EINVAL;
  }
  if (int st = bind_device(what, {out, rowptr, col, value, Xn, Xm, nu_out})) return st;
  return dispatch_float(dtype, [&](auto t0) {
    using T = decltype(t0);
    return dispatch_index(rowptr_dtype, [&](auto r0) {
      using RP = decltype(r0);
      return dispatch_index(col_dtype, [&](auto c0) {
        using CI = decltype(c0);
        return dispatch_dp(D, [&](auto dp) {
          constexpr int DP = decltype(dp)::value;
          auto rp = static_cast<const RP *>(rowptr);
          auto cp = static_cast<const CI *>(col);
          auto vp = static_cast<const T *>(value);
          auto xn = static_cast<const T *>(Xn);
          auto xm = static_cast<const T *>(Xm);
          auto op = static_cast<T *>(out);
          if constexpr (DP <= 16) {
            const int64_t blocks = (N + 7) / 8;
            scatter_cov_warp<T, RP, CI, DP><<<(unsigned)blocks, 256, 0, as_stream(stream)>>>(
                rp, cp, vp, xn, xm, op, N, M, (int)D, static_cast<T *>(nu_out), (T)nu0);
          } else {
            using C = CtaScatterCfg<T, DP>;
            auto kern = scatter_cov_cta<T, RP, CI, DP>;
            int st = set_smem(kern, C::smem);
            if (st) return st;
            kern<<<(unsigned)N, C::THREADS, C::smem, as_stream(stream)>>>(rp, cp, vp, xn, xm, op, N, M, (int)D,
                                                                          static_cast<T *>(nu_out), (T)nu0);
          }
          return check_launch(what);
        });
      });
    });
  });
}

extern "C" int lakde_W_inv(int dtype, const void *rowptr, int rowptr_dtype, const void *col, int col_dtype,
                           const void *value, const void *Xn, const void *Xm, void *out, int64_t N, int64_t M,
                           int64_t D, void *stream) {
  return scatter_cov_launch("W_inv", dtype, rowptr, rowptr_dtype, col, col_dtype, value, Xn, Xm, out, N, M, D,
                            nullptr, 0.0, stream);
}

extern "C" int lakde_mstep(int dtype, int64_t N, int64_t D, int64_t npts, const void *rowptr, int rowptr_dtype,
                           const void *col, int col_dtype, const void *r, const void *X, int64_t kernel_offset,
                           double nu_0, void *S, void *nu, void *stream) {
  if (kernel_offset < 0 || kernel_offset + N > npts) {
    clear_error();
    set_error("mstep: kernel rows [%lld, %lld) outside the %lld points", (long long)kernel_offset,
              (long long)(kernel_offset + N), (long long)npts);
    return LAKDE_EINVAL;
  }
  const size_t es = dtype == LAKDE_F64 ? 8 : 4;
  const void *Xn = X ? static_cast<const char *>(X) + (size_t)kernel_offset * (size_t)D * es : nullptr;
  return scatter_cov_launch("mstep", dtype, rowptr, rowptr_dtype, col, col_dtype, r, Xn, X, S, N, npts, D, nu, nu_0,
                            stream);
}
