// Backward of the predictive log density (lakde/local_adaptive_kde.py:200-223).
//
// With d = y - x_n, z = W_triu_n^T d = L_n^-1 d, Q = |z|^2, h_n = (nu_n + 1)/2,
// lp_ny = log_coeff_n - h_n log1p(Q), out_y = -log N + logsumexp_n lp_ny and
// the softmax weight w_ny = exp(lp_ny - out_y - log N), an upstream gradient
// g_y gives
//   d out / d y   = sum_n w_ny (-2 h_n / (1 + Q)) W_triu_n z          (score)
//   d out / d L_n = -(sum_y g_y w_ny) diag(1 / L_ii)
//                   + 2 h_n W_triu_n (sum_y c_ny z z^T),  c_ny = g_y w_ny / (1 + Q)
// (lower triangle).  The pair pass recomputes every quad form instead of
// storing the pair x D differences: it writes c_ny [N, Nq], the per-CTA row
// sums of g_y w_ny and the score partials; a dense scatter pass forms
// S_c[n] = sum_y c_ny d d^T, from which the host finishes d/dL_n with D x D
// products (sum_y c_ny z z^T = W_triu^T S_c W_triu).
#include "common.cuh"

namespace lakde {

template <typename T, int DP>
struct BwdCfg {
  static constexpr int QT = 128;
  static constexpr int KT = DP <= 16 ? 16 : (DP <= 32 ? 8 : 4);
  static constexpr int TS = Tri<T>::size(DP);
  // packed factor, centre, log coefficient, h
  static constexpr int per_kernel = ((TS + DP + 2 + Tri<T>::V - 1) / Tri<T>::V) * Tri<T>::V;
  static constexpr size_t smem = (size_t)KT * per_kernel * sizeof(T) + (size_t)KT * 4 * sizeof(T);
};

static int64_t bwd_chunk(int64_t N, int64_t Nq, int kt) {
  const int64_t q_tiles = (Nq + 127) / 128;
  const int64_t target = 148 * 4;
  int64_t nchunks = (target + q_tiles - 1) / q_tiles;
  if (nchunks < 1) nchunks = 1;
  int64_t chunk = (N + nchunks - 1) / nchunks;
  chunk = ((chunk + kt - 1) / kt) * kt;
  return chunk < kt ? kt : chunk;
}

// (U z)_i = sum_{j >= i} U[i][j] z_j for the packed upper factor (column j holds rows 0..j)
template <typename T, int DP>
__device__ __forceinline__ void upper_times(const T *__restrict__ sU, const T (&z)[DP], T (&out)[DP]) {
#pragma unroll
  for (int i = 0; i < DP; ++i) out[i] = T(0);
  int off = 0;
#pragma unroll
  for (int j = 0; j < DP; ++j) {
#pragma unroll
    for (int i = 0; i <= j; ++i) out[i] = fma(sU[off + i], z[j], out[i]);
    off += Tri<T>::col_len(j);
  }
}

template <typename T, int DP>
__global__ void __launch_bounds__(128) pred_bwd_pairs_kernel(
    const T *__restrict__ X, const T *__restrict__ W, const T *__restrict__ nu, const T *__restrict__ lcoef,
    const T *__restrict__ Y, const T *__restrict__ outp, const T *__restrict__ gout, T *__restrict__ cw,
    T *__restrict__ sw_part, T *__restrict__ score_part, int64_t N, int64_t Nq, int D, int64_t chunk, int64_t q_tiles,
    T log_n) {
  using C = BwdCfg<T, DP>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *sbase = reinterpret_cast<T *>(smem_raw);
  T *sred = sbase + C::KT * C::per_kernel;  // [KT][4] warp partials of sum_y g w
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int64_t qt = blockIdx.x % q_tiles;
  const int64_t ch = blockIdx.x / q_tiles;
  const int64_t q = qt * C::QT + tid;
  const bool qv = q < Nq;
  const int64_t n_begin = ch * chunk;
  const int64_t n_end = (n_begin + chunk < N) ? n_begin + chunk : N;

  T y[DP];
#pragma unroll
  for (int d = 0; d < DP; ++d) y[d] = (qv && d < D) ? Y[q * D + d] : T(0);
  const T ly = qv ? outp[q] + log_n : T(0);
  const T g = qv ? gout[q] : T(0);
  T score[DP];
#pragma unroll
  for (int d = 0; d < DP; ++d) score[d] = T(0);

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
    for (int k = 0; k < cnt; ++k) {
      const T *sk = sbase + k * C::per_kernel;
      const int64_t n = n0 + k;
      T delta[DP], z[DP];
#pragma unroll
      for (int d = 0; d < DP; ++d) delta[d] = y[d] - sk[C::TS + d];
      const T Q = quad_tri_z<T, DP>(sk, delta, z);
      const T h = sk[C::TS + DP + 1];
      const T lp = sk[C::TS + DP] - h * log1p(Q);
      const T w = qv ? exp(lp - ly) : T(0);
      const T c = g * w / (T(1) + Q);
      if (qv) cw[n * Nq + q] = c;
      // score: g w (-2 h / (1 + Q)) U z = -2 h c U z
      T uz[DP];
      upper_times<T, DP>(sk, z, uz);
      const T f = T(-2) * h * c;
#pragma unroll
      for (int d = 0; d < DP; ++d) score[d] = fma(f, uz[d], score[d]);
      // sum over this CTA's queries of g w for kernel n
      const T gw = warp_sum(g * w);
      if (lane == 0) sred[k * 4 + warp] = gw;
    }
    __syncthreads();
    for (int k = tid; k < cnt; k += C::QT) {
      const T s = sred[k * 4 + 0] + sred[k * 4 + 1] + sred[k * 4 + 2] + sred[k * 4 + 3];
      sw_part[qt * N + n0 + k] = s;
    }
  }
  if (qv) {
#pragma unroll
    for (int d = 0; d < DP; ++d)
      if (d < D) score_part[(ch * Nq + q) * D + d] = score[d];
  }
}

template <typename T>
__global__ void sum_parts_kernel(const T *__restrict__ parts, T *__restrict__ out, int64_t n, int64_t nparts) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  T s = T(0);
  for (int64_t p = 0; p < nparts; ++p) s += parts[p * n + i];
  out[i] = s;
}

// S_c[n] = sum_y c[n, y] (y - x_n)(y - x_n)^T over all queries; one CTA per
// kernel, threads own 4x4 blocks of the lower triangle, queries staged 64 at a
// time as centred differences.
template <typename T, int DP>
struct DenseScatterCfg {
  static constexpr int NB = DP < 4 ? 1 : DP / 4;
  static constexpr int NBLK = NB * (NB + 1) / 2;
  static constexpr int THREADS = ((NBLK + 31) / 32) * 32;
  static constexpr int CH = 64;
  static constexpr int LD = (DP < 4 ? 4 : DP) + 4;
};

template <typename T, int DP>
__global__ void dense_scatter_kernel(const T *__restrict__ cw, const T *__restrict__ X, const T *__restrict__ Y,
                                     T *__restrict__ S, int64_t N, int64_t Nq, int D) {
  using C = DenseScatterCfg<T, DP>;
  __shared__ __align__(16) T sd[C::CH][C::LD];
  __shared__ T sv[C::CH];
  __shared__ T sxn[C::LD];
  const int64_t n = blockIdx.x;
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
  for (int d = tid; d < C::LD; d += blockDim.x) sxn[d] = d < D ? X[n * D + d] : T(0);
  T acc[4][4];
#pragma unroll
  for (int p = 0; p < 4; ++p)
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[p][q] = T(0);
  for (int64_t base = 0; base < Nq; base += C::CH) {
    const int cnt = (int)((Nq - base) < C::CH ? (Nq - base) : C::CH);
    __syncthreads();
    for (int e = tid; e < C::CH * C::LD; e += blockDim.x) {
      const int pp = e / C::LD, d = e % C::LD;
      sd[pp][d] = (pp < cnt && d < D) ? Y[(base + pp) * D + d] - sxn[d] : T(0);
    }
    for (int pp = tid; pp < C::CH; pp += blockDim.x) sv[pp] = pp < cnt ? cw[n * Nq + base + pp] : T(0);
    __syncthreads();
    if (bi >= 0) {
      for (int pp = 0; pp < cnt; ++pp) {
        const T v = sv[pp];
        T a[4], b[4];
#pragma unroll
        for (int p = 0; p < 4; ++p) {
          a[p] = sd[pp][4 * bi + p];
          b[p] = v * sd[pp][4 * bj + p];
        }
#pragma unroll
        for (int p = 0; p < 4; ++p)
#pragma unroll
          for (int q = 0; q < 4; ++q) acc[p][q] = fma(b[q], a[p], acc[p][q]);
      }
    }
  }
  if (bi < 0) return;
  T *o = S + n * (int64_t)D * D;
#pragma unroll
  for (int p = 0; p < 4; ++p)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int i = 4 * bi + p, j = 4 * bj + q;
      if (i >= D || j > i) continue;
      o[i * D + j] = acc[p][q];
      o[j * D + i] = acc[p][q];
    }
}

static int bwd_kt(int dtype, int64_t D) {
  int kt = 0;
  dispatch_float(dtype, [&](auto t0) {
    using T = decltype(t0);
    return dispatch_dp(D, [&](auto dp) {
      kt = BwdCfg<T, decltype(dp)::value>::KT;
      return 0;
    });
  });
  return kt;
}

}  // namespace lakde

using namespace lakde;

extern "C" size_t lakde_log_pred_density_bwd_workspace(int dtype, int64_t N, int64_t Nq, int64_t D) {
  if (N <= 0 || Nq <= 0 || D < 1 || D > kMaxDim || (dtype != LAKDE_F32 && dtype != LAKDE_F64)) return 0;
  const int64_t chunk = bwd_chunk(N, Nq, bwd_kt(dtype, D));
  const int64_t nchunks = (N + chunk - 1) / chunk;
  const int64_t q_tiles = (Nq + 127) / 128;
  const size_t es = dtype == LAKDE_F32 ? 4 : 8;
  return (size_t)(q_tiles * N + nchunks * Nq * D) * es;
}

extern "C" int lakde_log_pred_density_bwd(int dtype, int64_t N, int64_t Nq, int64_t D, const void *X,
                                          const void *W_triu, const void *nu, const void *log_coeff, const void *Y,
                                          const void *out, const void *grad_out, void *grad_Y, void *cw, void *sw,
                                          void *S_c, void *workspace, size_t workspace_bytes, void *stream) {
  clear_error();
  if (N < 1 || Nq < 1 || D < 1) {
    set_error("log_pred_density_bwd: invalid sizes");
    return LAKDE_EINVAL;
  }
  const size_t need = lakde_log_pred_density_bwd_workspace(dtype, N, Nq, D);
  if (need == 0) {
    set_error("log_pred_density_bwd: unsupported dtype %d or D=%lld", dtype, (long long)D);
    return LAKDE_EUNSUPPORTED;
  }
  if (!workspace || workspace_bytes < need) {
    set_error("log_pred_density_bwd: workspace of %zu bytes needed, %zu given", need, workspace_bytes);
    return LAKDE_EINVAL;
  }
  if (!X || !W_triu || !nu || !log_coeff || !Y || !out || !grad_out || !grad_Y || !cw || !sw || !S_c) {
    set_error("log_pred_density_bwd: null pointer");
    return LAKDE_EINVAL;
  }
  if (int st = bind_device("log_pred_density_bwd",
                           {grad_Y, X, W_triu, nu, log_coeff, Y, out, grad_out, cw, sw, S_c, workspace}))
    return st;
  return dispatch_float(dtype, [&](auto t0) {
    using T = decltype(t0);
    return dispatch_dp(D, [&](auto dp) {
      constexpr int DP = decltype(dp)::value;
      using C = BwdCfg<T, DP>;
      const int64_t chunk = bwd_chunk(N, Nq, C::KT);
      const int64_t nchunks = (N + chunk - 1) / chunk;
      const int64_t q_tiles = (Nq + C::QT - 1) / C::QT;
      T *sw_part = static_cast<T *>(workspace);
      T *score_part = sw_part + q_tiles * N;
      auto kern = pred_bwd_pairs_kernel<T, DP>;
      if (C::smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::smem);
        if (e != cudaSuccess) {
          set_error("log_pred_density_bwd: %s", cudaGetErrorString(e));
          return (int)LAKDE_ECUDA;
        }
      }
      kern<<<(unsigned)(q_tiles * nchunks), C::QT, C::smem, as_stream(stream)>>>(
          static_cast<const T *>(X), static_cast<const T *>(W_triu), static_cast<const T *>(nu),
          static_cast<const T *>(log_coeff), static_cast<const T *>(Y), static_cast<const T *>(out),
          static_cast<const T *>(grad_out), static_cast<T *>(cw), sw_part, score_part, N, Nq, (int)D, chunk, q_tiles,
          (T)log((double)N));
      if (int st = check_launch("log_pred_density_bwd")) return st;
      sum_parts_kernel<T><<<(unsigned)((N + 255) / 256), 256, 0, as_stream(stream)>>>(sw_part, static_cast<T *>(sw),
                                                                                       N, q_tiles);
      if (int st = check_launch("log_pred_density_bwd_sw")) return st;
      sum_parts_kernel<T><<<(unsigned)((Nq * D + 255) / 256), 256, 0, as_stream(stream)>>>(
          score_part, static_cast<T *>(grad_Y), Nq * D, nchunks);
      if (int st = check_launch("log_pred_density_bwd_score")) return st;
      using SC = DenseScatterCfg<T, DP>;
      dense_scatter_kernel<T, DP><<<(unsigned)N, SC::THREADS, 0, as_stream(stream)>>>(
          static_cast<const T *>(cw), static_cast<const T *>(X), static_cast<const T *>(Y), static_cast<T *>(S_c), N,
          Nq, (int)D);
      return check_launch("log_pred_density_bwd_scatter");
    });
  });
}
