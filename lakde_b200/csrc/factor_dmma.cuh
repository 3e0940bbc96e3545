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
// NT is a template parameter so every tile offset is a compile-time constant
// and the independent tile products of one step can be issued back to back.
#pragma once

#include "common.cuh"

namespace lakde {
namespace dmma {

constexpr int TILE = 64;  // doubles per 8 x 8 tile

__host__ __device__ constexpr int tix(int I, int J) { return (I * (I + 1) / 2 + J) * TILE; }

__device__ __forceinline__ void mma(double &c0, double &c1, double a, double b) {
  // not volatile: the compiler may interleave independent tile products
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

__device__ __forceinline__ double afrag(const double *t, int s, int lane) { return t[(lane >> 2) * 8 + 4 * s + (lane & 3)]; }
// B = M
__device__ __forceinline__ double bfrag(const double *t, int s, int lane) { return t[(4 * s + (lane & 3)) * 8 + (lane >> 2)]; }
// B = M^T
__device__ __forceinline__ double bfrag_t(const double *t, int s, int lane) { return afrag(t, s, lane); }

__device__ __forceinline__ void load_c(const double *t, int lane, double &c0, double &c1) {
  const double2 v = *reinterpret_cast<const double2 *>(t + (lane >> 2) * 8 + 2 * (lane & 3));
  c0 = v.x;
  c1 = v.y;
}
__device__ __forceinline__ void store_c(double *t, int lane, double c0, double c1) {
  *reinterpret_cast<double2 *>(t + (lane >> 2) * 8 + 2 * (lane & 3)) = make_double2(c0, c1);
}

// B fragment (s) of the 8 x 8 tile whose C fragment the warp holds in (c0, c1):
// element (4 s + t % 4, t / 4) lives in lane 4 (4 s + t % 4) + (t / 4) / 2,
// component (t / 4) % 2.
__device__ __forceinline__ double c_to_b(double c0, double c1, int s, int lane) {
  const int src = 16 * s + 4 * (lane & 3) + (lane >> 3);
  const double v0 = __shfl_sync(0xffffffffu, c0, src);
  const double v1 = __shfl_sync(0xffffffffu, c1, src);
  return ((lane >> 2) & 1) ? v1 : v0;
}

// Cholesky and inverse of the 8 x 8 diagonal tile t (lower part), computed
// redundantly by every lane from broadcast shared-memory reads (no shuffles
// on the critical path).  On return t holds inv(L_KK) (lower, zero upper)
// and rdiag[k] = 1 / L_kk.  Returns false (warp-uniform) if a
// pivot is not positive.  If lt is given, L_KK (lower, zero upper) is written
// there too.
__device__ __forceinline__ bool diag_tile(double *t, double *rdiag, double *lt, int lane) {
  double a[36];  // packed lower, row i at i (i + 1) / 2
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j <= i; j += 2) {
      // pairs (j, j + 1); the element right of the diagonal of an even row is not kept
      const double2 v = *reinterpret_cast<const double2 *>(t + i * 8 + j);
      a[i * (i + 1) / 2 + j] = v.x;
      if (j + 1 <= i) a[i * (i + 1) / 2 + j + 1] = v.y;
    }
  bool ok = true;
  double rd[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const double piv = a[k * (k + 1) / 2 + k];
    ok = ok && (piv > 0.0);
    const double rs = rsqrt(piv > 0.0 ? piv : 1.0);
    rd[k] = rs;
    a[k * (k + 1) / 2 + k] = piv * rs;
#pragma unroll
    for (int i = k + 1; i < 8; ++i) a[i * (i + 1) / 2 + k] *= rs;
#pragma unroll
    for (int i = k + 1; i < 8; ++i)
#pragma unroll
      for (int j = k + 1; j <= i; ++j)
        a[i * (i + 1) / 2 + j] = fma(-a[i * (i + 1) / 2 + k], a[j * (j + 1) / 2 + k], a[i * (i + 1) / 2 + j]);
  }
  if (lane == 0 && lt) {
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
      for (int j = 0; j < 8; ++j) lt[i * 8 + j] = (j <= i) ? a[i * (i + 1) / 2 + j] : 0.0;
  }
  // X = L^-1 in place, column by column from the right: with the block below
  // and right of (j, j) already inverted, X_jj = 1 / L_jj and
  // X_ij = -X_jj sum_{k=j+1}^{i} X_ik L_kj (i > j)
#pragma unroll
  for (int j = 7; j >= 0; --j) {
    double col[8];
#pragma unroll
    for (int i = j + 1; i < 8; ++i) {
      double sacc = 0.0;
#pragma unroll
      for (int k = j + 1; k <= i; ++k) sacc = fma(a[i * (i + 1) / 2 + k], a[k * (k + 1) / 2 + j], sacc);
      col[i] = -sacc * rd[j];
    }
#pragma unroll
    for (int i = j + 1; i < 8; ++i) a[i * (i + 1) / 2 + j] = col[i];
    a[j * (j + 1) / 2 + j] = rd[j];
  }
  __syncwarp();
  // lane 0 writes, in pairs: every lane holds the same values
  if (lane == 0) {
#pragma unroll
    for (int i = 0; i < 8; ++i) {
#pragma unroll
      for (int j = 0; j < 8; j += 2)
        *reinterpret_cast<double2 *>(t + i * 8 + j) =
            make_double2((j <= i) ? a[i * (i + 1) / 2 + j] : 0.0, (j + 1 <= i) ? a[i * (i + 1) / 2 + j + 1] : 0.0);
    }
#pragma unroll
    for (int i = 0; i < 8; i += 2) *reinterpret_cast<double2 *>(rdiag + i) = make_double2(rd[i], rd[i + 1]);
  }
  __syncwarp();
  return ok;
}

// Blocked right-looking Cholesky of the tiled matrix M.  On return the
// diagonal tiles hold inv(L_KK) and the off-diagonal tiles L_IK; rdiag[i]
// holds 1 / L_ii.  If lout is given (row-major D x D), the
// factor L is written there as well (through the scratch tile).  The step loop runs at run time (small
// code); the tile loops inside a step are unrolled and predicated.
template <int NT, typename T>
__device__ __forceinline__ bool chol_blocked(double *M, double *scratch, double *rdiag, int lane, T *lout,
                                             int D) {
#pragma unroll 1
  for (int K = 0; K < NT; ++K) {
    double *dk = M + tix(K, K);
    if (!diag_tile(dk, rdiag + 8 * K, lout ? scratch : nullptr, lane)) return false;
    if (lout) {
      for (int e = lane; e < 64; e += 32) {
        const int i = 8 * K + e / 8, j = 8 * K + e % 8;
        if (i < D && j < D) lout[i * D + j] = (T)scratch[e];
      }
    }
    // panel: L_IK = A_IK inv(L_KK)^T
    const double b0 = bfrag_t(dk, 0, lane), b1 = bfrag_t(dk, 1, lane);
    double pc[NT][2];
#pragma unroll
    for (int I = 1; I < NT; ++I) {
      if (I > K) {
        const double *t = M + tix(I, 0) + K * TILE;
        pc[I][0] = 0.0;
        pc[I][1] = 0.0;
        mma(pc[I][0], pc[I][1], afrag(t, 0, lane), b0);
        mma(pc[I][0], pc[I][1], afrag(t, 1, lane), b1);
      }
    }
    __syncwarp();
#pragma unroll
    for (int I = 1; I < NT; ++I)
      if (I > K) store_c(M + tix(I, 0) + K * TILE, lane, pc[I][0], pc[I][1]);
    __syncwarp();
    // A fragments of the new panel (= B fragments of its transpose)
    double pa[NT][2];
#pragma unroll
    for (int I = 1; I < NT; ++I) {
      if (I > K) {
        pa[I][0] = afrag(M + tix(I, 0) + K * TILE, 0, lane);
        pa[I][1] = afrag(M + tix(I, 0) + K * TILE, 1, lane);
      }
    }
    // trailing update: A_IJ -= L_IK L_JK^T, K < J <= I (each lane touches its own C elements)
#pragma unroll
    for (int J = 1; J < NT; ++J) {
      if (J > K) {
        // keeps the loads of one column of tiles together (register pressure)
        asm volatile("" ::: "memory");
#pragma unroll
        for (int I = J; I < NT; ++I) {
          double *t = M + tix(I, J);
          double c0, c1;
          load_c(t, lane, c0, c1);
          mma(c0, c1, -pa[I][0], pa[J][0]);
          mma(c0, c1, -pa[I][1], pa[J][1]);
          store_c(t, lane, c0, c1);
        }
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
// off-diagonal tiles L_IJ; on return the tiles hold X = L^-1.  Row block by
// row block: X_IJ = -inv(L_II) sum_{K=J}^{I-1} L_IK X_KJ needs the finished
// rows above and the L tiles of row I only, so the I tiles of row I are
// independent; their products are interleaved (K outer, J inner) and they are
// stored together once all of them are computed.
template <int NT>
__device__ __forceinline__ void trtri_blocked(double *M, int lane) {
#pragma unroll 1
  for (int I = 1; I < NT; ++I) {
    const double *rowI = M + tix(I, 0);
    double c[NT][2];
#pragma unroll
    for (int J = 0; J < NT; ++J) {
      c[J][0] = 0.0;
      c[J][1] = 0.0;
    }
#pragma unroll 1
    for (int K = 0; K < I; ++K) {
      const double a0 = afrag(rowI + K * TILE, 0, lane), a1 = afrag(rowI + K * TILE, 1, lane);
      const double *rowK = M + (K * (K + 1) / 2) * TILE;
#pragma unroll
      for (int J = 0; J < NT - 1; ++J) {
        if (J <= K) {
          mma(c[J][0], c[J][1], a0, bfrag(rowK + J * TILE, 0, lane));
          mma(c[J][0], c[J][1], a1, bfrag(rowK + J * TILE, 1, lane));
        }
      }
    }
    const double *di = rowI + I * TILE;
    const double n0 = -afrag(di, 0, lane), n1 = -afrag(di, 1, lane);
    double xo[NT][2];
#pragma unroll
    for (int J = 0; J < NT - 1; ++J) {
      if (J < I) {
        xo[J][0] = 0.0;
        xo[J][1] = 0.0;
        mma(xo[J][0], xo[J][1], n0, c_to_b(c[J][0], c[J][1], 0, lane));
        mma(xo[J][0], xo[J][1], n1, c_to_b(c[J][0], c[J][1], 1, lane));
      }
    }
    __syncwarp();
#pragma unroll
    for (int J = 0; J < NT - 1; ++J)
      if (J < I) store_c(M + tix(I, 0) + J * TILE, lane, xo[J][0], xo[J][1]);
    __syncwarp();
  }
}

}  // namespace dmma
}  // namespace lakde
