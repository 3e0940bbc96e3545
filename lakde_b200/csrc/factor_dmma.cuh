// Warp-level FP64 blocked Cholesky with its triangular inverse on the FP64
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

// Cholesky and inverse of the 8 x 8 diagonal tile t (lower part): the
// Cholesky redundantly on every lane from broadcast shared-memory reads (no
// shuffles on its rsqrt chain), the inverse one column per lane.  On return
// t holds inv(L_KK) (lower, zero upper)
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
  // X = L^-1 by forward substitution, one column per lane (j = lane % 8):
  // X_ij = (δ_ij - sum_{k<i} L_ik X_kj) / L_ii, zero above the diagonal.  The
  // lanes run the same instructions on their own column (36 FP64 operations
  // instead of the whole inverse on every lane); X_(i-1)j enters last, so the
  // chain is one FMA and one multiply per row.
  const int jc = lane & 7;
  double x[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    double acc = (i == jc) ? 1.0 : 0.0;
#pragma unroll
    for (int k = 0; k < i; ++k) acc = fma(-a[i * (i + 1) / 2 + k], x[k], acc);
    x[i] = acc * rd[i];
  }
  __syncwarp();
  if (lane < 8) {
#pragma unroll
    for (int i = 0; i < 8; ++i) t[i * 8 + jc] = x[i];
  }
  if (lane == 0) {
#pragma unroll
    for (int i = 0; i < 8; i += 2) *reinterpret_cast<double2 *>(rdiag + i) = make_double2(rd[i], rd[i + 1]);
  }
  __syncwarp();
  return ok;
}

// Blocked right-looking Cholesky of the tiled matrix M with the inverse
// X = L^-1 formed in the same sweep.  Forward substitution L X = I by row
// blocks gives X_KK = inv(L_KK), X_KJ = inv(L_KK) X'_KJ and, for the rows
// below, X'_IJ -= L_IK X_KJ, so step K:
//   1. factorises the diagonal tile (inv(L_KK) in place of A_KK);
//   2. forms the panel L_IK = A_IK inv(L_KK)^T (I > K) and, independently,
//      the finished row X_KJ = inv(L_KK) X'_KJ (J < K);
//   3. per column J: the trailing update A_IJ -= L_IK L_JK^T (J > K) or the
//      substitution update X'_IJ -= L_IK X_KJ (J <= K, I > K), both with the
//      panel's A fragments.
// Column K of L is consumed in step K, and X'_IK (= -L_IK X_KK) takes its
// tile.  On return the tiles hold X (diagonal tiles inv(L_KK)) and rdiag[i]
// holds 1 / L_ii.  If lout is given (row-major D x D), the factor L is
// written there as well.  If l0t is given (the lower 8 x 8 tiles of a lower
// triangular L0 in FP32, same tile order), each lane's share of
// ||X L0||_F^2 is added to trace_acc: row K of Z = X L0 is
// Z_KA = sum_{A <= J <= K} X_KJ L0_JA, formed column by column beside the
// substitution update once row K of X is final.  The step loop runs at run time (small code); the
// tile loops inside a step are unrolled and predicated.
template <int NT, typename T>
__device__ __forceinline__ bool chol_inv_blocked(double *M, double *scratch, double *rdiag, int lane, T *lout,
                                                 int D, const float *l0t, double &trace_acc) {
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
    // fragments of inv(L_KK): B = inv(L_KK)^T for the panel, A = inv(L_KK)
    // for the finished row of X (the same elements)
    const double g0 = afrag(dk, 0, lane), g1 = afrag(dk, 1, lane);
    double pc[NT][2], xr[NT][2];
#pragma unroll
    for (int I = 1; I < NT; ++I) {
      if (I > K) {
        const double *t = M + tix(I, 0) + K * TILE;
        pc[I][0] = 0.0;
        pc[I][1] = 0.0;
        mma(pc[I][0], pc[I][1], afrag(t, 0, lane), g0);
        mma(pc[I][0], pc[I][1], afrag(t, 1, lane), g1);
      }
    }
#pragma unroll
    for (int J = 0; J < NT - 1; ++J) {
      if (J < K) {
        const double *t = M + tix(K, J);
        xr[J][0] = 0.0;
        xr[J][1] = 0.0;
        mma(xr[J][0], xr[J][1], g0, bfrag(t, 0, lane));
        mma(xr[J][0], xr[J][1], g1, bfrag(t, 1, lane));
      }
    }
    __syncwarp();
#pragma unroll
    for (int I = 1; I < NT; ++I)
      if (I > K) store_c(M + tix(I, 0) + K * TILE, lane, pc[I][0], pc[I][1]);
#pragma unroll
    for (int J = 0; J < NT - 1; ++J)
      if (J < K) store_c(M + tix(K, J), lane, xr[J][0], xr[J][1]);
    __syncwarp();
    if (lout) {
      for (int I = K + 1; I < NT; ++I)
        for (int e = lane; e < 64; e += 32) {
          const int i = 8 * I + e / 8, j = 8 * K + e % 8;
          if (i < D && j < D) lout[i * D + j] = (T)M[tix(I, K) + e];
        }
    }
    // A fragments of the panel (= B fragments of its transpose); the tiles
    // (I, K) are rewritten with X'_IK below, after every lane has read them
    double pa[NT][2];
#pragma unroll
    for (int I = 1; I < NT; ++I) {
      if (I > K) {
        pa[I][0] = afrag(M + tix(I, K), 0, lane);
        pa[I][1] = afrag(M + tix(I, K), 1, lane);
      }
    }
    __syncwarp();
    double z[NT][2];
#pragma unroll
    for (int A = 0; A < NT; ++A) z[A][0] = z[A][1] = 0.0;
#pragma unroll
    for (int J = 0; J < NT; ++J) {
      // keeps the loads of two columns of tiles together (register pressure;
      // the second column's loads overlap the first one's products)
      if ((J & 1) == 0) asm volatile("" ::: "memory");
      if (J > K) {
        // trailing update: A_IJ -= L_IK L_JK^T, J <= I
#pragma unroll
        for (int I = J; I < NT; ++I) {
          double *t = M + tix(I, J);
          double c0, c1;
          load_c(t, lane, c0, c1);
          mma(c0, c1, -pa[I][0], pa[J][0]);
          mma(c0, c1, -pa[I][1], pa[J][1]);
          store_c(t, lane, c0, c1);
        }
      } else {
        const double *xk = M + tix(K, J);
        if (K + 1 < NT) {
          // substitution update: X'_IJ -= L_IK X_KJ, I > K (X'_IK starts at 0)
          const double b0 = bfrag(xk, 0, lane), b1 = bfrag(xk, 1, lane);
#pragma unroll
          for (int I = 1; I < NT; ++I) {
            if (I > K) {
              double *t = M + tix(I, J);
              double c0 = 0.0, c1 = 0.0;
              if (J < K) load_c(t, lane, c0, c1);
              mma(c0, c1, -pa[I][0], b0);
              mma(c0, c1, -pa[I][1], b1);
              store_c(t, lane, c0, c1);
            }
          }
        }
        if (l0t) {
          // trace row K: Z_KA += X_KJ L0_JA, A <= J (L0 tile: local row
          // lane % 4 (+ 4), local column lane / 4)
          const double a0 = afrag(xk, 0, lane), a1 = afrag(xk, 1, lane);
#pragma unroll
          for (int A = 0; A <= J; ++A) {
            const float *tk = l0t + (J * (J + 1) / 2 + A) * 64 + (lane & 3) * 8 + (lane >> 2);
            mma(z[A][0], z[A][1], a0, (double)tk[0]);
            mma(z[A][0], z[A][1], a1, (double)tk[32]);
          }
        }
      }
    }
    if (l0t) {
      // ||Z_K.||^2: squares per tile, then a tree over the tiles
      double sq[NT];
#pragma unroll
      for (int A = 0; A < NT; ++A) sq[A] = fma(z[A][0], z[A][0], z[A][1] * z[A][1]);
#pragma unroll
      for (int w = 1; w < NT; w *= 2)
#pragma unroll
        for (int A = 0; A + w < NT; A += 2 * w) sq[A] += sq[A + w];
      trace_acc += sq[0];
    }
    __syncwarp();
  }
  return true;
}

}  // namespace dmma
}  // namespace lakde
