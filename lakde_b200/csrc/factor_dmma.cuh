// Warp-level FP64 blocked Cholesky, triangular inverse and trace on the FP64
// tensor cores (mma.sync m8n8k4 f64), for the batched posterior factorisation
// with 16 <= D <= 64.
//
// A D x D symmetric matrix (padded to DP = 8 NT with the identity) lives in
// shared memory as its NT (NT + 1) / 2 lower 8 x 8 tiles, tile (I, J) at index
// I (I + 1) / 2 + J, each row-major.  Fragments of m8n8k4 (lane t):
//   A (8 x 4, row-major)  a = M[t / 4][4 s + t % 4]
//   B (4 x 8, col-major)  b = M[4 s + t % 4][t / 4]      (B = M)
//                         b = M[t / 4][4 s + t % 4]      (B = M^T)
//   C (8 x 8)             c0, c1 = M[t / 4][2 (t % 4) + {0, 1}]
#pragma once

#include "common.cuh"

namespace lakde {
namespace dmma {

constexpr int TILE = 64;  // doubles per 8 x 8 tile

__device__ __forceinline__ int tix(int I, int J) { return (I * (I + 1) / 2 + J) * TILE; }

__device__ __forceinline__ void mma(double &c0, double &c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

__device__ __forceinline__ double afrag(const double *t, int s, int lane) { return t[(lane >> 2) * 8 + 4 * s + (lane & 3)]; }
// B = M
__device__ __forceinline__ double bfrag(const double *t, int s, int lane) { return t[(4 * s + (lane & 3)) * 8 + (lane >> 2)]; }
// B = M^T
__device__ __forceinline__ double bfrag_t(const double *t, int s, int lane) { return afrag(t, s, lane); }

__device__ __forceinline__ void load_c(const double *t, int lane, double &c0, double &c1) {
  const int o = (lane >> 2) * 8 + 2 * (lane & 3);
  c0 = t[o];
  c1 = t[o + 1];
}
__device__ __forceinline__ void store_c(double *t, int lane, double c0, double c1) {
  const int o = (lane >> 2) * 8 + 2 * (lane & 3);
  t[o] = c0;
  t[o + 1] = c1;
}

// Cholesky of the lower part of one 8 x 8 tile in place (lanes 0..7 own rows);
// returns false (warp-uniform) if a pivot is not positive.  The upper part is
// zeroed.
__device__ __forceinline__ bool chol_tile(double *t, int lane) {
  double r[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) r[j] = (lane < 8 && j <= lane) ? t[lane * 8 + j] : 0.0;
  bool ok = true;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const double piv = __shfl_sync(0xffffffffu, r[k], k);
    ok = ok && (piv > 0.0);
    const double lkk = sqrt(piv > 0.0 ? piv : 1.0);
    if (lane == k) r[k] = lkk;
    if (lane > k && lane < 8) r[k] = r[k] / lkk;
#pragma unroll
    for (int j = k + 1; j < 8; ++j) {
      const double ljk = __shfl_sync(0xffffffffu, r[k], j);
      if (lane >= j && lane < 8) r[j] -= r[k] * ljk;
    }
  }
  __syncwarp();
  if (lane < 8) {
#pragma unroll
    for (int j = 0; j < 8; ++j) t[lane * 8 + j] = (j <= lane) ? r[j] : 0.0;
  }
  __syncwarp();
  return ok;
}

// inv(L) of a lower 8 x 8 tile (lanes 0..7 own columns), written to `out`
// (lower, zero upper).  `t` is read only.
__device__ __forceinline__ void inv_tile(const double *t, double *out, int lane) {
  double x[8];
  const int c = lane;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    double s = (i == c) ? 1.0 : 0.0;
#pragma unroll
    for (int k = 0; k < i; ++k) s -= t[i * 8 + k] * ((k >= c) ? x[k] : 0.0);
    x[i] = (i >= c) ? s / t[i * 8 + i] : 0.0;
  }
  __syncwarp();
  if (lane < 8) {
#pragma unroll
    for (int i = 0; i < 8; ++i) out[i * 8 + c] = x[i];
  }
  __syncwarp();
}

// Blocked right-looking Cholesky of the tiled matrix M (NT tiles per side).
// On return the diagonal tiles hold inv(L_KK) and the off-diagonal tiles
// L_IK; the diagonal of L is saved in ldiag[0..8 NT).  If lout is given
// (row-major D x D, ld), the factor L is written there as well.
template <typename T>
__device__ __forceinline__ bool chol_blocked(double *M, double *scratch, double *ldiag, int NT, int lane, T *lout,
                                             int D) {
  for (int K = 0; K < NT; ++K) {
    double *dk = M + tix(K, K);
    if (!chol_tile(dk, lane)) return false;
    if (lane < 8) ldiag[8 * K + lane] = dk[lane * 8 + lane];
    if (lout) {
      for (int e = lane; e < 64; e += 32) {
        const int i = 8 * K + e / 8, j = 8 * K + e % 8;
        if (i < D && j < D) lout[i * D + j] = (T)(j <= i ? dk[e] : 0.0);
      }
    }
    inv_tile(dk, scratch, lane);
    for (int e = lane; e < 64; e += 32) dk[e] = scratch[e];
    __syncwarp();
    // panel: L_IK = A_IK inv(L_KK)^T
    for (int I = K + 1; I < NT; ++I) {
      double *t = M + tix(I, K);
      double c0 = 0.0, c1 = 0.0;
#pragma unroll
      for (int s = 0; s < 2; ++s) mma(c0, c1, afrag(t, s, lane), bfrag_t(dk, s, lane));
      __syncwarp();
      store_c(t, lane, c0, c1);
      __syncwarp();
    }
    // trailing update: A_IJ -= L_IK L_JK^T, K < J <= I
    for (int J = K + 1; J < NT; ++J) {
      const double *lj = M + tix(J, K);
      for (int I = J; I < NT; ++I) {
        const double *li = M + tix(I, K);
        double *t = M + tix(I, J);
        double c0, c1;
        load_c(t, lane, c0, c1);
#pragma unroll
        for (int s = 0; s < 2; ++s) mma(c0, c1, -afrag(li, s, lane), bfrag_t(lj, s, lane));
        store_c(t, lane, c0, c1);
      }
    }
    __syncwarp();
    if (lout) {
      for (int I = K + 1; I < NT; ++I)
        for (int e = lane; e < 64; e += 32) {
          const int i = 8 * I + e / 8, j = 8 * K + e % 8;
          if (i < D && j < D) lout[i * D + j] = (T)M[tix(I, K) + e];
        }
    }
  }
  return true;
}

// In-place blocked inverse: on entry the diagonal tiles hold inv(L_II) and the
// off-diagonal tiles L_IJ; on return the tiles hold X = L^-1.
__device__ __forceinline__ void trtri_blocked(double *M, double *scratch, int NT, int lane) {
  for (int J = 0; J < NT; ++J) {
    for (int I = J + 1; I < NT; ++I) {
      // acc = sum_{K=J}^{I-1} L_IK X_KJ
      double c0 = 0.0, c1 = 0.0;
      for (int K = J; K < I; ++K) {
        const double *l = M + tix(I, K);
        const double *x = M + tix(K, J);
#pragma unroll
        for (int s = 0; s < 2; ++s) mma(c0, c1, afrag(l, s, lane), bfrag(x, s, lane));
      }
      store_c(scratch, lane, c0, c1);
      __syncwarp();
      // X_IJ = -inv(L_II) acc
      const double *di = M + tix(I, I);
      double d0 = 0.0, d1 = 0.0;
#pragma unroll
      for (int s = 0; s < 2; ++s) mma(d0, d1, -afrag(di, s, lane), bfrag(scratch, s, lane));
      __syncwarp();
      store_c(M + tix(I, J), lane, d0, d1);
      __syncwarp();
    }
  }
}

}  // namespace dmma
}  // namespace lakde
