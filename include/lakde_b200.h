/*
 * lakde_b200 — C ABI of the B200 (sm_100a) kernels for the variational-inference
 * hot path of the locally adaptive KDEs of falkaer/lakde.
 *
 * Conventions shared by every entry point:
 *  - plain device pointers and sizes; no framework types cross this boundary;
 *  - `stream` is a cudaStream_t passed as void* (NULL = legacy default stream);
 *    every call is asynchronous on that stream and never synchronises;
 *  - dtype codes are the lakde_dtype values below; value arrays are row-major
 *    and contiguous unless strides are passed explicitly;
 *  - the caller owns and allocates every buffer, outputs included, exactly as the
 *    reference's torch ops receive a preallocated `out`;
 *  - the return value is a lakde_status; on failure lakde_last_error() gives a
 *    message (per host thread).  Invalid indices found on the device do not fault:
 *    the affected output rows are written as NaN.
 *
 * References are file:line inside the reference project (falkaer/lakde).
 */
#ifndef LAKDE_B200_H_
#define LAKDE_B200_H_

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define LAKDE_API __attribute__((visibility("default")))
#else
#define LAKDE_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  LAKDE_F32 = 0,
  LAKDE_F64 = 1,
  LAKDE_I32 = 2,
  LAKDE_I64 = 3
} lakde_dtype;

typedef enum {
  LAKDE_OK = 0,
  LAKDE_EINVAL = 1,      /* bad sizes, pointers or strides */
  LAKDE_EDTYPE = 2,      /* unsupported dtype combination */
  LAKDE_ECUDA = 3,       /* a CUDA runtime call failed */
  LAKDE_EUNSUPPORTED = 4 /* shape outside what the kernels implement */
} lakde_status;

/* Message describing the last failed call on this host thread ("" if none). */
LAKDE_API const char *lakde_last_error(void);

/* Version of this ABI (incremented on any signature change). */
LAKDE_API int lakde_abi_version(void);

/* Largest data dimensionality D the factorisation and sparse kernels accept. */
LAKDE_API int lakde_max_dim(void);

/*
 * Launch choices of kernels that have more than one equivalent form; every
 * choice gives the same results, only the speed differs.  An autotuner times
 * them on the caller's data and keeps the fastest, per knob and class of D
 * (D <= 16, <= 32, <= 48, <= 64; process-wide, read at each launch).  No
 * counterpart in the reference.
 *   LAKDE_TUNE_FACTOR: 0 = the FP64 factorisation with two warps per block;
 *                      1 = one warp per block, 11 blocks per SM, for calls
 *                          that stage no T and write no L (else 0 is used).
 *   LAKDE_TUNE_ROWS:   0 = tensor-core rows from the caller's work queue;
 *                      1 = a static stride over the grid (the queue ignored).
 *   LAKDE_TUNE_VI_ROWS: 0 = lakde_vi_rows with a kernel row's pairs on two
 *                          lanes and its FP64 posterior on one lane per row;
 *                      1 = one thread per kernel row.
 */
typedef enum {
  LAKDE_TUNE_FACTOR = 0,
  LAKDE_TUNE_ROWS = 1,
  LAKDE_TUNE_VI_ROWS = 2,
  LAKDE_TUNE_KNOBS = 3
} lakde_tune_knob;
LAKDE_API int lakde_tuning_set(int knob, int64_t D, int value);
LAKDE_API int lakde_tuning_get(int knob, int64_t D);

/* ------------------------------------------------------------------------- */
/* The three ops of the reference extension (same argument meaning).         */
/* ------------------------------------------------------------------------- */

/*
 * CSR row pointer from a sorted row-index vector: out[i] = #{p : ind[p] < i},
 * i = 0..M.  Replaces lakde::ind2ptr_cuda(Tensor ind, int M, Tensor out)
 * (csrc/cuda/convert_cuda.cu:46-65, registered :67-68; Python wrapper
 * lakde/kernels.py:93-100).  ind: I32/I64 [nnz]; out: I32/I64 [M+1].
 * nnz == 0 writes zeros, as the reference does.
 */
LAKDE_API int lakde_ind2ptr(const void *ind, int ind_dtype, int64_t nnz, int64_t M,
                  void *out, int out_dtype, void *stream);

/*
 * Dense Cholesky quad forms out[n,m] = || W_triu[n]^T (Xm[m] - Xn[n]) ||^2.
 * Replaces lakde::chol_quad_form_cuda(W_triu, Xn, Xm, out)
 * (csrc/cuda/chol_quad_form.cu:78-114; wrapper lakde/kernels.py:115-120).
 * W_triu [N,D,D] must be upper triangular; entries below the diagonal are not
 * read.  Strides are in elements (W: 3, Xn/Xm/out: 2), like the reference.
 * dtype: F32 or F64.
 */
LAKDE_API int lakde_chol_quad_form(int dtype, const void *W_triu, const int64_t *W_strides,
                         const void *Xn, const int64_t *Xn_strides,
                         const void *Xm, const int64_t *Xm_strides, void *out,
                         const int64_t *out_strides, int64_t N, int64_t M,
                         int64_t D, void *stream);

/*
 * Responsibility-weighted scatter covariance (the M-step),
 * out[n] = sum_{p in row n} value[p] (Xm[col[p]] - Xn[n]) (Xm[col[p]] - Xn[n])^T,
 * written as a full symmetric D x D matrix.  Replaces
 * lakde::W_inv_cuda(rowptr, col, value, Xn, Xm, out)
 * (csrc/cuda/W_inv_cuda.cu:70-137; wrapper lakde/kernels.py:102-113).
 * rowptr: I32/I64 [N+1]; col: I32/I64 [nnz]; value: dtype [nnz];
 * Xn [N,D], Xm [M,D], out [N,D,D] contiguous.  dtype: F32 or F64.  A row with
 * a column index outside [0, M) or a decreasing rowptr is written as NaN.
 */
LAKDE_API int lakde_W_inv(int dtype, const void *rowptr, int rowptr_dtype, const void *col,
                int col_dtype, const void *value, const void *Xn,
                const void *Xm, void *out, int64_t N, int64_t M, int64_t D,
                void *stream);

/* ------------------------------------------------------------------------- */
/* New ops of the hot path.                                                   */
/* ------------------------------------------------------------------------- */

/*
 * Batched posterior factorisation in FP64 with the per-matrix jitter ladder.
 * For every n:
 *   A_n = scale_n * P_n + S_n,   scale_n = nu_0 * a_n / b_n (if a, b given, else 1)
 *   L_n = chol(A_n + jitter_n I); on failure jitter_n is re-laddered from zero
 *         through eps * (2^(k+1) - 1), k = 0..31, and info_n = -1 if none works
 *   W_triu_n = L_n^-T (upper),  logdet_W_n = 2 sum_i log W_triu_n[i,i]
 *   trace_n  = || T_n^T W_triu_n ||_F^2   (if T given)
 * Restates lakde/local_adaptive_kde.py:83-96 (calc_posterior),
 * lakde/linalg_util.py:109-170 (stabilize_/stabilized_cholesky), :49-52
 * (tril_inverse), :30-37 (chol_logdet, chol_mm_trace).
 * P (optional) and T (optional) are [D,D] blocks with a batch stride in
 * elements (0 = one matrix shared by all n).  T_lower != 0 declares every
 * T_n lower triangular (its entries above the diagonal are then not read).
 * S [N,D,D] contiguous.
 * jitter [N] is read and updated in place.  Outputs: W_triu [N,D,D],
 * L [N,D,D] (optional), logdet_W [N], info [N] (int32: 0 ok, -1 ladder failed),
 * trace [N] (optional).  All value arrays have `dtype` (F32/F64); a, b, nu_0
 * too.  D <= lakde_max_dim().  W_cores (optional, float32 only, 16-byte
 * aligned): W_triu_n also as the W cores of the tensor-core kernels
 * (lakde_pack_w_cores layout; NaN for a matrix whose ladder failed).
 */
LAKDE_API int lakde_posterior_factor(int dtype, int64_t N, int64_t D, const void *S,
                           const void *P, int64_t P_batch_stride,
                           const void *nu_0, const void *a, const void *b,
                           void *jitter, double eps, void *W_triu, void *L,
                           void *logdet_W, int32_t *info, const void *T,
                           int64_t T_batch_stride, int T_lower, void *trace,
                           void *W_cores, void *stream);

/*
 * Fused-path M-step: the scatter covariance of lakde_W_inv for kernels
 * n = kernel_offset .. kernel_offset + N - 1 of X (Xn = X[kernel_offset:]) and
 * nu_n = nu_0 + sum_{p in row n} r[p] in the same pass.  Restates
 * lakde/local_adaptive_kde.py:66-81 (calc_posterior_contribs).
 * rowptr [N+1], col [nnz] (I32/I64), r [nnz], X [npts,D], S [N,D,D], nu [N].
 */
LAKDE_API int lakde_mstep(int dtype, int64_t N, int64_t D, int64_t npts,
                          const void *rowptr, int rowptr_dtype, const void *col,
                          int col_dtype, const void *r, const void *X,
                          int64_t kernel_offset, double nu_0, void *S, void *nu,
                          void *stream);

/*
 * Sparse-pair E-step numerators.  For kernel n in [0, N) and every pair p of
 * its CSR row (rowptr over the N kernels, col = point index into X[npts,D]):
 *   logrho[p] = 0.5 (mvdigamma(nu_n / 2, D) + D log 2 + logdet_W_n)
 *               - 0.5 nu_n || W_triu_n^T (X[col[p]] - X[n + kernel_offset]) ||^2
 * and logrho[p] = -inf for the self pair col[p] == n + kernel_offset.
 * Restates lakde/local_adaptive_kde.py:36-44 and :126-128 on a pair pattern.
 */
LAKDE_API int lakde_estep_logrho(int dtype, int64_t N, int64_t D, int64_t npts,
                       const void *rowptr, int rowptr_dtype, const void *col,
                       int col_dtype, const void *X, int64_t kernel_offset,
                       const void *W_triu, const void *nu, const void *logdet_W,
                       void *logrho, void *stream);

/*
 * One VI iteration's per-kernel work for D <= 8 in a single pass, one thread
 * per kernel row (kernels are the points 0..N-1 of X[npts,D]):
 *   nu_n = nu_0 + sum_p r_p and S_n = sum_p r_p (x_m - x_n)(x_m - x_n)^T
 *   L_n = chol(nu_0 a_n / b_n P_n + S_n + jitter_n I) in FP64 with the ladder of
 *         lakde_posterior_factor (info_n = -1 when it fails)
 *   logdet_W_n = -2 sum log L_ii; mm_n = nu_n ||L_n^-1 T_n||_F^2 (if T given;
 *         = nu_n chol_mm_trace(T_n, W_triu_n)) and then b_n = b_0 + nu_0 mm_n / 2
 *   logrho_p = 0.5 (mvdigamma(nu_n/2, D) + D log 2 + logdet_W_n)
 *              - nu_n / 2 ||L_n^-1 (x_m - x_n)||^2  (-inf on the self pair)
 * Restates lakde/local_adaptive_kde.py:66-96 and :36-44 and
 * lakde/local_knn_kde.py:220-236 for the batch schedule.  rowptr I64 [N+1],
 * col I32 [nnz], order I32 [N] (visiting order, may be NULL), r / logrho [nnz],
 * P and T [D,D] blocks with batch strides (0 = shared), a, b (in/out), jitter
 * (in/out), nu, logdet_W, mm [N] (mm may be NULL), info [N].  Row n is the
 * kernel centred on point n + kernel_offset of X (a shard's rows; npts >=
 * N + kernel_offset); the per-kernel arrays are indexed by n.
 */
LAKDE_API int lakde_vi_rows(int dtype, int64_t N, int64_t D, int64_t npts,
                            const void *rowptr, const void *col,
                            const void *order, const void *r, const void *X,
                            int64_t kernel_offset, double nu_0,
                            const void *P, int64_t P_batch_stride,
                            const void *T, int64_t T_batch_stride,
                            const void *a, void *b, double b_0, void *jitter,
                            double eps, void *nu, void *logdet_W, void *mm,
                            int32_t *info, void *logrho, void *stream);

/*
 * Mixed-precision tensor-core kernels (tcgen05.mma kind::tf32), float32
 * values, D <= 64.  The centred differences (x_m - x_n, and for the M-step
 * sqrt(r) (x_m - x_n)) and W_triu are split as x = hi + lo with
 * hi = tf32(x), lo = tf32(x - hi) (round to nearest); every product is
 * hi*hi + lo*hi + hi*lo with fp32 accumulation in tensor memory, within about
 * 2^-22 of the exact product (close to plain fp32 arithmetic).
 *
 * Point rows are moved by bulk copies, so X (and Y) must have 16-byte
 * aligned rows: base 16-byte aligned, row stride ldx (elements) a multiple
 * of 4 and >= D rounded up to 4; columns past D are never used.  Rows are
 * visited in `order` (may be NULL) through an atomic work queue: `queue`
 * is one device int32 the call resets to zero on `stream` before the launch
 * (NULL: a static stride over the grid).  *err is set to 1 if a completion
 * wait of the kernel times out; the affected rows are then left unwritten.
 * No counterpart in the reference (its ops run on CUDA cores, lakde/kernels.py).
 */

/*
 * "W cores": X_n = L_n^-1 = W_triu_n^T (lower) as the K-major 8 x 4 core
 * matrices of the tensor-core B operand, split into tf32 parts: x = hi + lo
 * with hi = x rounded to the nearest tf32 (ties away from zero) and lo = the
 * same rounding of x - hi.  With NT = 8-row blocks (those of
 * lakde_tile_count for D > 8, one block for D <= 8), per kernel, for column
 * block J = 0..NT-1 the hi parts of row blocks I = J..NT-1, then their lo
 * parts, each block as two cores (columns 8J..8J+3, then 8J+4..8J+7) of 32
 * floats: element X[i][j] at 32 ((j % 8) / 4) + 4 (i % 8) + j % 4 of its
 * block.  Zero outside D and above the diagonal.  lakde_w_cores_floats(D)
 * floats per kernel.
 */
LAKDE_API size_t lakde_w_cores_floats(int64_t D);

/*
 * Test hook of the bounded completion waits (no counterpart in the reference):
 * lakde_estep_tc's kernel on the given inputs (float32, no order, no queue)
 * with the first staged tile of each CTA expecting 16 bytes more than its
 * copies deliver.  Every issued copy lands, so nothing stays in flight; the
 * wait gives up after its time limit (1.5 s), *err becomes 1 and the kernel
 * frees its tensor memory and returns.
 */
LAKDE_API int lakde_tc_wait_timeout_probe(int64_t N, int64_t D, int64_t npts,
                                          const void *rowptr, const void *col,
                                          const void *X, int64_t ldx,
                                          const void *W_cores, const void *nu,
                                          const void *logdet_W, void *logrho,
                                          int32_t *err, void *stream);

/* W cores of N kernels from W_triu [N, D, D] (dense, upper; float32). */
LAKDE_API int lakde_pack_w_cores(int dtype, int64_t N, int64_t D,
                                 const void *W_triu, void *W_cores,
                                 void *stream);

/*
 * Tensor-core E-step: the logrho of lakde_estep_logrho for rows n = 0..N-1,
 * row n being kernel n + kernel_offset of X [npts, ldx], W_triu given as W
 * cores (16-byte aligned).  Restates lakde/local_adaptive_kde.py:36-44 on a
 * pair pattern.
 */
LAKDE_API int lakde_estep_tc(int dtype, int64_t N, int64_t D, int64_t npts,
                             const void *rowptr, const void *col,
                             const void *order, const void *X, int64_t ldx,
                             int64_t kernel_offset, const void *W_cores,
                             const void *nu, const void *logdet_W, void *logrho,
                             int32_t *queue, int32_t *err, void *stream);

/*
 * Tensor-core M-step: S_n and nu_n of lakde_mstep for rows n = 0..N-1, row n
 * being kernel n + kernel_offset of X [npts, ldx] (S symmetric up to the
 * order of the fp32 accumulation).  lower_only != 0 writes only the lower
 * triangle (j <= i) of each S_n and leaves the rest untouched (all
 * lakde_posterior_factor reads).  Restates lakde/local_adaptive_kde.py:66-81.
 */
LAKDE_API int lakde_mstep_tc(int dtype, int64_t N, int64_t D, int64_t npts,
                             const void *rowptr, const void *col,
                             const void *order, const void *r, const void *X,
                             int64_t ldx, int64_t kernel_offset, double nu_0,
                             void *S, void *nu, int lower_only, int32_t *queue,
                             int32_t *err, void *stream);

/*
 * Per-point normaliser, responsibilities and rebalance over a pair pattern
 * given point-major: pairs of point m are pos[cptr[m] .. cptr[m+1]) (indices
 * into logrho / r).  mode 0 (initial pass): c_m = logsumexp_n logrho.
 * mode 1 (update): c_m = logaddexp(logsubexp(c_m, log(rsum_m) + c_m), logsumexp).
 * Then r = exp(logrho - c_m), zeroed where r <= threshold; s_m = max(sum r, eps);
 * c_m += log s_m; r *= clamp(1 / s_m, tiny, max); rsum_m = sum of the new r.
 * Restates lakde/local_adaptive_kde.py:120-145 (partial_expectation_step at
 * block_size = N) and :156-181 (rebalance_responsibilities_).
 * cptr: I64 [npts+1]; pos: I32/I64 [nnz]; logrho, r: dtype [nnz];
 * c, rsum: dtype [npts] (in/out).
 */
LAKDE_API int lakde_estep_normalise(int dtype, int64_t npts, const void *cptr,
                          const void *pos, int pos_dtype, const void *logrho,
                          void *r, void *c, void *rsum, int mode,
                          double threshold, void *stream);

/*
 * lakde_estep_normalise split into four stages for kernels sharded over
 * devices (each device holds the pairs of its kernels; cptr / pos index its
 * own pairs, over all npts points).  The caller reduces over the devices
 * between stages: red by max after stage 0, red2 by sum after stages 1 and 2,
 * rsum by sum after stage 3.
 *   stage 0: red[m]  = max_local logrho
 *   stage 1: red2[m] = sum_local exp(logrho - red[m])
 *   stage 2: c_new from (c, rsum, red + log red2) as in lakde_estep_normalise;
 *            red[m] = c_new, red2[m] = sum_local of the thresholded r
 *   stage 3: c[m] = c_new + log(max(red2, eps)), r = r / red2 (clamped) on the
 *            local pairs, rsum[m] = sum_local of the new r
 * With one device (no reduction) the result equals lakde_estep_normalise.
 * No counterpart of its own in the reference, whose rebalance runs on one
 * device (lakde/local_adaptive_kde.py:120-181).  red, red2: dtype [npts].
 */
LAKDE_API int lakde_estep_normalise_stage(int dtype, int stage, int64_t npts,
                                          const void *cptr, const void *pos,
                                          int pos_dtype, const void *logrho,
                                          void *r, void *c, void *rsum, void *red,
                                          void *red2, int mode, double threshold,
                                          void *stream);

/*
 * Student-t log coefficients of the predictive density:
 *   log_coeff_n = lgamma((nu_n+1)/2) - lgamma((nu_n+1-D)/2) + logdet_W_n / 2
 *                 - D/2 log(pi), evaluated in FP64 (lakde/local_adaptive_kde.py:209-214).
 */
LAKDE_API int lakde_pred_coeff(int dtype, int64_t N, int64_t D, const void *nu,
                     const void *logdet_W, void *log_coeff, void *stream);

/* Workspace bytes lakde_log_pred_density needs for N kernels and Nq queries. */
LAKDE_API size_t lakde_log_pred_density_workspace(int dtype, int64_t N, int64_t Nq,
                                        int64_t D);

/*
 * Predictive log density of Nq queries under the N-kernel Student-t mixture:
 *   out[q] = -log N + logsumexp_n [ log_coeff_n
 *            - (nu_n + 1)/2 log1p(|| W_triu_n^T (Y[q] - X[n]) ||^2) ]
 * (lakde/local_adaptive_kde.py:200-223).  workspace: device buffer of at least
 * lakde_log_pred_density_workspace() bytes.
 */
LAKDE_API int lakde_log_pred_density(int dtype, int64_t N, int64_t Nq, int64_t D,
                           const void *X, const void *W_triu, const void *nu,
                           const void *log_coeff, const void *Y, void *out,
                           void *workspace, size_t workspace_bytes,
                           void *stream);

/* ------------------------------------------------------------------------- */
/* Tiled per-kernel matrices (8 < D <= 64, float32).                          */
/* ------------------------------------------------------------------------- */
/*
 * With DP = D rounded up to 16, 24, 32, 48 or 64 and NT = DP / 8, a matrix is
 * kept as its NT (NT + 1) / 2 lower 8 x 8 tiles, tile (I, J), J <= I, at
 * index I (I + 1) / 2 + J, each 64 floats row-major, zero outside D x D and
 * above the diagonal.  "SP" interleaves, per kernel and tile, the S tile
 * then the P tile (128 floats per tile): the bytes of a tile pair are exactly
 * those of the FP64 tile the factorisation builds from it, so one bulk copy
 * per matrix brings both operands in.  No counterpart in the reference (its
 * matrices are dense [N, D, D]).
 */
/* Number of tiles NT (NT + 1) / 2 for dimension D (0 if D is out of range). */
LAKDE_API int64_t lakde_tile_count(int64_t D);

/*
 * dst[n * dst_batch_stride + t * dst_tile_stride + dst_offset + e] = element
 * e of tile t of src[n] ([D, D] blocks src_batch_stride elements apart).
 */
LAKDE_API int lakde_pack_tiles(int dtype, int64_t N, int64_t D, const void *src,
                               int64_t src_batch_stride, void *dst,
                               int64_t dst_batch_stride, int64_t dst_tile_stride,
                               int64_t dst_offset, void *stream);

/*
 * lakde_mstep_tc with S_n written as tiles into the S halves of SP (per
 * kernel 128 * tiles floats); nu as in lakde_mstep_tc.  8 < D <= 64.
 */
LAKDE_API int lakde_mstep_tc_tiled(int dtype, int64_t N, int64_t D, int64_t npts,
                                   const void *rowptr, const void *col,
                                   const void *order, const void *r,
                                   const void *X, int64_t ldx,
                                   int64_t kernel_offset, double nu_0, void *SP,
                                   void *nu, int32_t *queue, int32_t *err,
                                   void *stream);

/*
 * lakde_posterior_factor from tiled inputs: A_n = nu_0 a_n / b_n P_n + S_n
 * with S_n and P_n from SP, and the trace term from the lower triangular T_n
 * as tiles (T_tiles, 64 * tiles floats per kernel, may be NULL).  float32,
 * 8 < D <= 64, SP and T_tiles 16-byte aligned.  Outputs as in
 * lakde_posterior_factor (no L), W_triu dense [N, D, D], X_tiles:
 * X_n = L_n^-1 = W_triu_n^T as lower tiles (64 * tiles floats per kernel)
 * and / or W_cores (16-byte aligned, lakde_w_cores_floats(D) floats per
 * kernel; NaN for a failed matrix); any two may be NULL.  info_n = -2 marks a matrix whose
 * input copy did not complete within the wait limit.
 */
LAKDE_API int lakde_posterior_factor_tiled(int dtype, int64_t N, int64_t D,
                                           const void *SP, const void *nu_0,
                                           const void *a, const void *b,
                                           void *jitter, double eps,
                                           void *W_triu, void *X_tiles,
                                           void *W_cores, void *logdet_W,
                                           int32_t *info, const void *T_tiles,
                                           void *trace, void *stream);

/* Workspace bytes lakde_weighted_gram needs for dimension D. */
LAKDE_API size_t lakde_weighted_gram_workspace(int64_t D);

/*
 * out [D, D] (float64, full symmetric) = sum_n w_n W_triu_n W_triu_n^T over
 * N kernels, W_triu [N, D, D] upper (dtype F32/F64) and w [N]: the
 * hierarchical model's shared-precision sum (lakde/local_hierarchical_kde.py:
 * 293-297) in FP64 without a float64 copy of the factors; deterministic
 * (fixed reduction order).
 */
LAKDE_API int lakde_weighted_gram(int dtype, int64_t N, int64_t D,
                                  const void *W_triu, const void *w,
                                  double *out, void *workspace,
                                  size_t workspace_bytes, void *stream);

/*
 * Selection half of the exact kNN graph (lakde/utils.py:77-116: cdist +
 * topk per row block, the point itself excluded at :104-105 unless
 * include_self).  dist [nb, N] (float64, row-major) holds the squared
 * distances of points row0 .. row0 + nb - 1 to all N points of X [N, D]
 * (float64), e.g. |a|^2 + |b|^2 - 2ab from a library GEMM.  Per row: the
 * k + 8 smallest entries (one pass, a shared-memory candidate buffer with a
 * running threshold) are re-ranked by exact float64 differences, and the k
 * nearest by (exact distance, index) go to out_idx [nb, k] (idx_dtype I32 /
 * I64) and, if out_dist is given, their distances to out_dist [nb, k]
 * (dist_dtype F32 / F64).  k <= N (include_self) or N - 1; candidates must
 * fit in 200 KB of shared memory (k up to 15,352).
 */
LAKDE_API int lakde_knn_select(const void *dist, int64_t nb, int64_t N,
                               int64_t row0, const void *X, int64_t D,
                               int include_self, int64_t k, int idx_dtype,
                               void *out_idx, int dist_dtype, void *out_dist,
                               void *stream);

/* Workspace bytes lakde_knn_elbo needs. */
LAKDE_API size_t lakde_knn_elbo_workspace(void);

/*
 * ELBO of LocalKNearestKDE in FP64 (lakde/local_knn_kde.py:256-341, terms
 * :24-47) from the per-kernel a, b, nu, logdet_W, logdet_sigma_0,
 * mm = nu * trace [N] and the per-point normaliser c [N], written to *out (one
 * double on the device).  Deterministic reduction order.
 */
/*
 * The same sums over separate counts: the kernel terms of kernels
 * 0..n_kernels-1 (a .. mm indexed by kernel) plus the point terms of points
 * 0..n_points-1 (c), plus `tail` (lakde_knn_elbo passes -N log(N - 1)).
 * A sharded caller sums the kernel terms of its rows over the ranks and adds
 * the point terms once.  Either count may be 0 (its arrays may then be NULL).
 */
LAKDE_API int lakde_knn_elbo_parts(int dtype, int64_t n_kernels, int64_t n_points,
                                   int64_t D, const void *a, const void *b,
                                   const void *nu, const void *logdet_W,
                                   const void *logdet_sigma_0, const void *mm,
                                   const void *c, double a_0, double b_0,
                                   double nu_0, double tail, void *workspace,
                                   size_t workspace_bytes, double *out,
                                   void *stream);

LAKDE_API int lakde_knn_elbo(int dtype, int64_t N, int64_t D, const void *a,
                             const void *b, const void *nu, const void *logdet_W,
                             const void *logdet_sigma_0, const void *mm,
                             const void *c, double a_0, double b_0, double nu_0,
                             void *workspace, size_t workspace_bytes,
                             double *out, void *stream);

/* Workspace bytes lakde_log_pred_density_tc needs (float32, D <= 64). */
LAKDE_API size_t lakde_log_pred_density_tc_workspace(int64_t N, int64_t Nq,
                                                     int64_t D);

/*
 * lakde_log_pred_density with the quad forms on the tensor cores (the tf32
 * hi / lo kernels above; queries in blocks of 2048, every query of a block
 * against every kernel), float32 values, D <= 64, X [N, ldx] and Y [Nq, ldy]
 * with 16-byte aligned rows, W_triu given as W cores
 * (lakde/local_adaptive_kde.py:200-223).  *err as for the tensor-core E-step.
 */
LAKDE_API int lakde_log_pred_density_tc(int dtype, int64_t N, int64_t Nq,
                                        int64_t D, const void *X, int64_t ldx,
                                        const void *W_cores, const void *nu,
                                        const void *log_coeff, const void *Y,
                                        int64_t ldy, void *out, void *workspace,
                                        size_t workspace_bytes, int32_t *err,
                                        void *stream);

/* Workspace bytes lakde_log_pred_density_bwd needs. */
LAKDE_API size_t lakde_log_pred_density_bwd_workspace(int dtype, int64_t N,
                                                      int64_t Nq, int64_t D);

/*
 * Backward of lakde_log_pred_density for an upstream gradient g [Nq] (new;
 * the reference's log_pred_density, lakde/local_adaptive_kde.py:200-223, is
 * not differentiable).  With z = W_triu_n^T (y - x_n), Q = |z|^2,
 * h_n = (nu_n + 1)/2 and softmax weights w_ny over kernels (recomputed from
 * the forward output `out`), writes
 *   grad_Y [Nq, D]  = sum_n g_y w_ny (-2 h_n / (1 + Q)) W_triu_n z      (score)
 *   cw [N, Nq]      = g_y w_ny / (1 + Q)
 *   sw [N]          = sum_y g_y w_ny
 *   S_c [N, D, D]   = sum_y cw_ny (y - x_n)(y - x_n)^T
 * from which d/dL_n = 2 h_n W_triu_n W_triu_n^T S_c W_triu_n - sw_n diag(1/L_ii)
 * (lower part) for the Cholesky factor L_n = W_triu_n^-T.  Quad forms are
 * recomputed, never stored per pair and dimension.
 */
LAKDE_API int lakde_log_pred_density_bwd(int dtype, int64_t N, int64_t Nq,
                                         int64_t D, const void *X,
                                         const void *W_triu, const void *nu,
                                         const void *log_coeff, const void *Y,
                                         const void *out, const void *grad_out,
                                         void *grad_Y, void *cw, void *sw,
                                         void *S_c, void *workspace,
                                         size_t workspace_bytes, void *stream);

/*
 * lakde_log_pred_density without any device allocation.  This entry point has
 * no counterpart in the reference.  It is for callers that cannot call
 * cudaMalloc: hosts that own all device memory themselves (a framework's
 * caching allocator, a plugin sandbox) or that forbid device allocation once
 * they are running.  Same arguments and result as lakde_log_pred_density
 * minus the workspace, which comes from a 16 MiB array built into the library
 * (each GPU that loads the library holds it until the process exits).  Calls
 * that would need more than 16 MiB of scratch (see
 * lakde_log_pred_density_workspace) are rejected with LAKDE_EINVAL; split the
 * queries.  The first call on each device looks up the array's device address
 * with that device current and keeps it for the life of the process, so it is
 * stale after a cudaDeviceReset (or any re-creation of the primary context):
 * do not use this entry point across a device reset.  Make the first call
 * before any stream capture.  All calls share the array: calls that overlap
 * on the GPU race on it.
 */
LAKDE_API int lakde_log_pred_density_noalloc(int dtype, int64_t N, int64_t Nq,
                                             int64_t D, const void *X,
                                             const void *W_triu, const void *nu,
                                             const void *log_coeff,
                                             const void *Y, void *out,
                                             void *stream);

#ifdef __cplusplus
}
#endif

#endif /* LAKDE_B200_H_ */
