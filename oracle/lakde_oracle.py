"""CPU oracle for the lakde variational-inference hot path.

TEST INFRASTRUCTURE ONLY.  This module is the checker, never the product:
only ``tests/``, ``__graft_entry__.smoke()`` and the CPU legs of ``bench.py``
(``cpu_baseline`` and ``--impl reference``) may import it.  The product path
(``lakde_b200``) never calls into it and fails loudly when its CUDA library
is missing.

It restates, in numpy (float32 or float64 arrays), the algorithm of the
reference implementation falkaer/lakde (paths below are relative to that
project):

* the three custom ops of ``lakde/kernels.py`` (ind2ptr, chol_quad_form,
  calc_W_inv);
* the kNN graph and the COO responsibility pattern it seeds
  (``lakde/utils.py``, ``lakde/sparse_util.py``);
* the jittered Cholesky ladder (``lakde/linalg_util.py``);
* block coordinate-ascent VI for ``LocalKNearestKDE`` and
  ``LocalHierarchicalKDE`` with the dense E-step, the running normaliser and
  the rebalance step (``lakde/local_adaptive_kde.py``,
  ``lakde/local_knn_kde.py``, ``lakde/local_hierarchical_kde.py``);
* ``log_pred_density`` and the ELBO.

Optionally the E-step is restricted to a fixed candidate pair pattern (pairs
outside it get log rho = -inf); with the all-pairs pattern this is the
reference algorithm itself.

Parity is pinned: ``tests/test_oracle_golden.py`` checks every function here
against golden vectors produced by running the reference code itself
(``tests/golden/make_golden.py``), in float32 and float64.
"""

import math

import numpy as np
import scipy.sparse
import scipy.special

LOG2 = math.log(2.0)
LOGPI = math.log(math.pi)


# ---------------------------------------------------------------------------
# special functions (lakde/linalg_util.py:8-26)
# ---------------------------------------------------------------------------


def lgamma(a):
    """log Gamma evaluated in float64 and cast back (lakde/linalg_util.py:8-9)."""
    a = np.asarray(a)
    return scipy.special.gammaln(a.astype(np.float64)).astype(a.dtype)


def mvlgamma(a, D):
    """Multivariate log Gamma (lakde/linalg_util.py:13-18)."""
    a = np.asarray(a)
    i = np.arange(1, D + 1, dtype=a.dtype)
    terms = lgamma(a[..., None] + (1 - i) / 2)
    return (D * (D - 1) / 4 * LOGPI + terms.sum(-1)).astype(a.dtype)


def mvdigamma(a, D):
    """Multivariate digamma sum_i psi(a + (1 - i)/2) (lakde/linalg_util.py:22-26)."""
    a = np.asarray(a)
    i = np.arange(1, D + 1, dtype=a.dtype)
    terms = scipy.special.digamma((a[..., None] + (1 - i) / 2).astype(np.float64))
    return terms.astype(a.dtype).sum(-1).astype(a.dtype)


def chol_logdet(L):
    """2 * sum(log(diag(L))) (lakde/linalg_util.py:30-31)."""
    return 2 * np.log(np.diagonal(L, axis1=-2, axis2=-1)).sum(-1)


def chol_mm_trace(L, R):
    """||L^T R||_F^2 = tr(L L^T R R^T) (lakde/linalg_util.py:35-37)."""
    LR = np.swapaxes(L, -1, -2) @ R
    return (LR * LR).sum(axis=(-1, -2))


def logsubexp(a, b):
    """a + log1p(max(-exp(b - a), -1)) (lakde/linalg_util.py:41-42)."""
    with np.errstate(invalid="ignore", over="ignore"):
        return a + np.log1p(np.maximum(-np.exp(b - a), -1.0).astype(np.asarray(a).dtype))


def logsumexp0(x):
    """logsumexp over axis 0 with the all -inf column mapping to -inf."""
    m = x.max(axis=0)
    ms = np.where(np.isfinite(m), m, 0).astype(x.dtype)
    with np.errstate(divide="ignore"):
        return (np.log(np.exp(x - ms).sum(axis=0)) + ms).astype(x.dtype)


def xlogx(x):
    with np.errstate(divide="ignore", invalid="ignore"):
        return np.where(x == 0, 0, x * np.log(np.where(x == 0, 1, x))).astype(x.dtype)


def tril_inverse(L):
    """Inverse of lower-triangular L (lakde/linalg_util.py:49-52)."""
    D = L.shape[-1]
    eye = np.broadcast_to(np.eye(D, dtype=L.dtype), L.shape)
    return np.linalg.solve(L, eye).astype(L.dtype)


# ---------------------------------------------------------------------------
# the three custom ops (lakde/kernels.py:11-39; csrc/cuda/*.cu)
# ---------------------------------------------------------------------------


def ind2ptr(row, M, dtype=np.int64):
    """CSR row pointer of a sorted row-index vector.

    out[i] = number of entries with row < i, for i in [0, M] (lakde/kernels.py:11-17,
    csrc/cuda/convert_cuda.cu:30-44).
    """
    row = np.asarray(row)
    return np.searchsorted(row, np.arange(M + 1), side="left").astype(dtype)


def chol_quad_form(W_triu, Xn, Xm):
    """Q[n, m] = ||W_triu[n]^T (Xm[m] - Xn[n])||^2 (lakde/kernels.py:20-23).

    Only the upper triangle of each W_triu[n] is read, as the CUDA kernel does
    (csrc/cuda/chol_quad_form.cu:33, loop cj <= ci); for exactly upper-triangular
    inputs this equals the dense fallback.
    """
    U = np.triu(W_triu)
    diff = Xm[None, :, :] - Xn[:, None, :]
    Y = np.einsum("nji,nmj->nmi", U, diff, optimize=True)
    return (Y * Y).sum(-1)


def _rows_of(rowptr):
    rowptr = np.asarray(rowptr, dtype=np.int64)
    return np.repeat(np.arange(len(rowptr) - 1), np.diff(rowptr))


def calc_W_inv(rowptr, col, value, Xn, Xm):
    """S[n] = sum_c value[c] (Xm[col[c]] - Xn[n]) (Xm[col[c]] - Xn[n])^T.

    Restates lakde/kernels.py:26-39 and csrc/cuda/W_inv_cuda.cu:7-68 (one row of
    the CSR per kernel n; the output is symmetric).
    """
    N, D = Xn.shape
    rowptr = np.asarray(rowptr, dtype=np.int64)
    nnz = int(rowptr[-1] - rowptr[0])
    col = np.asarray(col, dtype=np.int64)[rowptr[0] : rowptr[0] + nnz]
    value = np.asarray(value)[rowptr[0] : rowptr[0] + nnz]
    rows = _rows_of(rowptr - rowptr[0])
    diff = Xm[col] - Xn[rows]
    outer = (value[:, None, None] * diff[:, :, None]) * diff[:, None, :]
    agg = scipy.sparse.csr_matrix(
        (np.ones(nnz, dtype=np.float64), (rows, np.arange(nnz))), shape=(N, nnz)
    )
    out = agg @ outer.reshape(nnz, D * D).astype(np.float64)
    out = np.asarray(out).reshape(N, D, D).astype(value.dtype)
    return out


# ---------------------------------------------------------------------------
# kNN graph and the responsibility pattern (lakde/utils.py:77-116,
# lakde/sparse_util.py:8-54)
# ---------------------------------------------------------------------------


def knn_graph(X, k, include_self=False, block=1024):
    """k nearest neighbours of every row of X, nearest first.

    Distances are exact squared euclidean distances in float64 and ties are
    broken by the lower index; this is the order-defining oracle for
    lakde/utils.py:77-116 (which uses cdist + topk).  Without include_self the
    point itself is excluded (utils.py:104-105).
    """
    X64 = np.asarray(X, dtype=np.float64)
    N = X64.shape[0]
    out = np.empty((N, k), dtype=np.int64)
    idx_all = np.arange(N)
    for s in range(0, N, block):
        Xb = X64[s : s + block]
        d2 = ((Xb[:, None, :] - X64[None, :, :]) ** 2).sum(-1)
        if not include_self:
            d2[np.arange(len(Xb)), s + np.arange(len(Xb))] = np.inf
        if k < N:
            part = np.argpartition(d2, k, axis=1)[:, : k + 1]
        else:
            part = np.broadcast_to(idx_all, d2.shape)
        for r in range(len(Xb)):
            cand = part[r]
            dc = d2[r, cand]
            order = np.lexsort((cand, dc))
            out[s + r] = cand[order][:k]
    return out


def knn_pattern(graph, block_size=None):
    """COO pairs (kernel n, point m) for every n in the kNN list of m.

    Restates lakde/sparse_util.py:8-54 (graph_to_slices): row = neighbour n
    (relative to its kernel block), col = point m (global), sorted by row.
    Within a row the reference order is that of an unstable argsort; here the
    canonical order is ascending col.  Returns a list of [2, nnz_b] int arrays.
    """
    graph = np.asarray(graph)
    N, K = graph.shape
    B = N if block_size is None else min(block_size, N)
    rows = graph.reshape(-1).astype(np.int64)
    cols = np.repeat(np.arange(N), K)
    order = np.lexsort((cols, rows))
    rows, cols = rows[order], cols[order]
    ptr = ind2ptr(rows, N)
    out = []
    for s in range(0, N, B):
        e = min(s + B, N)
        a, b = ptr[s], ptr[e]
        out.append(np.stack([rows[a:b] - s, cols[a:b]]))
    return out


def batched_knn_cov(X, X_self, graph):
    """Sigma0[n] = 1/K sum_k (x_k - x_n)(x_k - x_n)^T over the kNN list of n.

    lakde/utils.py:40-65 with include_self=False, self_center=True.
    """
    K = graph.shape[1]
    diff = X[graph] - X_self[:, None, :]
    return (np.swapaxes(diff, -1, -2) @ diff / K).astype(X.dtype)


def cov(X):
    """Unbiased sample covariance in float64 (lakde/utils.py:28-37)."""
    X64 = np.asarray(X, dtype=np.float64)
    Xc = X64 - X64.mean(0, keepdims=True)
    return Xc.T @ Xc / (X64.shape[0] - 1)


# ---------------------------------------------------------------------------
# jittered Cholesky (lakde/linalg_util.py:91-170)
# ---------------------------------------------------------------------------


def cholesky_info(A):
    """Batched lower Cholesky with a LAPACK-style info code.

    info[b] = 0 on success, else j + 1 for the first column j whose pivot is not
    positive (or is NaN); restates the contract of torch.linalg.cholesky_ex used
    by lakde/linalg_util.py:100, 137-139.
    """
    A = np.asarray(A)
    single = A.ndim == 2
    if single:
        A = A[None]
    B, D, _ = A.shape
    L = np.zeros_like(A)
    info = np.zeros(B, dtype=np.int64)
    for j in range(D):
        s = A[:, j, j] - (L[:, j, :j] ** 2).sum(-1)
        bad = ~(s > 0)
        info = np.where((info == 0) & bad, j + 1, info)
        d = np.sqrt(np.where(info == 0, s, 1)).astype(A.dtype)
        L[:, j, j] = d
        if j + 1 < D:
            num = A[:, j + 1 :, j] - np.einsum("bik,bk->bi", L[:, j + 1 :, :j], L[:, j, :j])
            L[:, j + 1 :, j] = num / d[:, None]
    if single:
        return L[0], info[0]
    return L, info


def _with_jitter(X, jitter):
    out = np.array(X, copy=True)
    D = X.shape[-1]
    out[..., np.arange(D), np.arange(D)] += np.asarray(jitter)[..., None]
    return out


def stabilize(X, eps):
    """Per-matrix jitter eps * (2^(k+1) - 1) for the first k making X PD.

    lakde/linalg_util.py:109-126; raises after 32 doublings.
    """
    jitter = np.zeros(X.shape[:-2], dtype=X.dtype)
    mask = np.ones(X.shape[:-2], dtype=bool)
    for k in range(32):
        jitter[mask] += np.asarray(eps * 2.0**k, dtype=X.dtype)
        _, info = cholesky_info(_with_jitter(X, jitter))
        mask = np.asarray(info) != 0
        if not mask.any():
            return jitter
    raise RuntimeError("Stabilization did not converge")


def stabilized_cholesky(X, jitter=None, eps=None):
    """Cholesky of X + diag(jitter), re-laddering the jitter of failed matrices.

    lakde/linalg_util.py:129-170.  Returns (L, jitter).
    """
    X = np.asarray(X)
    if eps is None:
        eps = np.finfo(X.dtype).eps
    if jitter is not None and np.count_nonzero(jitter) != 0:
        L, info = cholesky_info(_with_jitter(X, jitter))
    else:
        L, info = cholesky_info(X)
    info = np.atleast_1d(info)
    if not info.any():
        return L, jitter
    if jitter is None:
        jitter = np.zeros(X.shape[:-2], dtype=X.dtype)
    else:
        jitter = np.array(jitter, copy=True)
    mask = info != 0
    if X.ndim == 2:
        jitter = stabilize(X[None], eps)[0]
    else:
        jitter[mask] = stabilize(X[mask], eps)
    return stabilized_cholesky(X, jitter, eps)


# ---------------------------------------------------------------------------
# E-step helpers (lakde/local_adaptive_kde.py:36-44)
# ---------------------------------------------------------------------------


def log_rho_const(nu, logdet_W, D):
    """0.5 * E[log|Lambda_n|] (lakde/local_adaptive_kde.py:37-40)."""
    dt = np.asarray(nu).dtype
    return (0.5 * (mvdigamma(nu / 2, D) + D * LOG2 + logdet_W)).astype(dt)


def calc_log_rho_block(X_test, X_train, nu, W_triu, logdet_W):
    """log rho[n, m] = const_n - nu_n / 2 * Q[n, m] (lakde/local_adaptive_kde.py:36-44)."""
    D = X_test.shape[-1]
    Q = chol_quad_form(W_triu, X_train, X_test)
    return (Q * (-0.5 * nu)[:, None] + log_rho_const(nu, logdet_W, D)[:, None]).astype(
        X_test.dtype
    )


# ---------------------------------------------------------------------------
# block VI models (lakde/local_adaptive_kde.py, lakde/local_knn_kde.py,
# lakde/local_hierarchical_kde.py)
# ---------------------------------------------------------------------------


class _AdaptiveOracle:
    """Shared state and steps of the locally adaptive models.

    ``candidates``: optional boolean [N, N] mask (kernel n, point m) restricting
    the E-step to a fixed pair pattern; None means all pairs (the reference).
    """

    def __init__(self, nu_0=None, k=20, block_size=512, a_0=1e-6, b_0=1e-6, candidates=None):
        self.nu_0_arg = nu_0
        self.k_arg = k
        self.block_size = block_size
        self.a_0_arg = a_0
        self.b_0_arg = b_0
        self.candidates = candidates
        self.iter_steps = 0

    # -- blocks -----------------------------------------------------------
    def _blocks(self, N):
        return [(s, min(s + self.block_size, N)) for s in range(0, N, self.block_size)]

    def _posterior_contribs(self, X, bi):
        """S and nu of block bi from its COO (lakde/local_adaptive_kde.py:66-81)."""
        s, e = self._blocks(len(X))[bi]
        (row, col), val = self.rnm_blocks[bi]
        rowptr = ind2ptr(row, e - s)
        S = calc_W_inv(rowptr, col, val, X[s:e], X)
        nu = np.full(e - s, self.nu_0, dtype=X.dtype)
        np.add.at(nu, row.astype(np.int64), val)
        return S, nu

    def _posterior(self, bi, N, sigma_0, S):
        """W_triu = chol(nu0 E[tau] Sigma0 + S)^-T (lakde/local_adaptive_kde.py:83-96)."""
        s, e = self._blocks(N)[bi]
        expect_tau = self.a[s:e] / self.b[s:e]
        W_inv = (sigma_0.astype(S.dtype) * (self.nu_0 * expect_tau)[:, None, None]).astype(S.dtype)
        W_inv = W_inv + S
        L, jit = stabilized_cholesky(W_inv, self.W_inv_jitter[s:e], eps=self.eps)
        if jit is not None:
            self.W_inv_jitter[s:e] = jit
        return np.swapaxes(tril_inverse(L), -1, -2)

    def _mask_block(self, log_rho, bi, bj, N):
        s, e = self._blocks(N)[bi]
        js, je = self._blocks(N)[bj]
        if bi == bj:
            idx = np.arange(e - s)
            log_rho[idx, idx] = -np.inf
        if self.candidates is not None:
            log_rho[~self.candidates[s:e, js:je]] = -np.inf
        return log_rho

    def _expectation(self, X, bi, W_triu, nu, update_normalization, threshold):
        """Dense E-step of block bi (lakde/local_adaptive_kde.py:98-154)."""
        N, D = X.shape
        blocks = self._blocks(N)
        s, e = blocks[bi]
        logdet_W = chol_logdet(W_triu)
        c = self.rnm_log_consts
        old_c = c
        if update_normalization:
            c = c.copy()
            (row, col), val = self.rnm_blocks[bi]
            old_sums = np.zeros(N, dtype=X.dtype)
            np.add.at(old_sums, col.astype(np.int64), val)
            with np.errstate(divide="ignore"):
                old_contrib = np.log(old_sums) + old_c
        rows, cols, vals = [], [], []
        for bj, (js, je) in enumerate(blocks):
            log_rho = calc_log_rho_block(X[js:je], X[s:e], nu, W_triu, logdet_W)
            log_rho = self._mask_block(log_rho, bi, bj, N)
            if update_normalization:
                new_contrib = logsumexp0(log_rho)
                c[js:je] = np.logaddexp(logsubexp(old_c[js:je], old_contrib[js:je]), new_contrib)
            with np.errstate(invalid="ignore"):
                r = np.exp(log_rho - c[js:je][None, :]).astype(X.dtype)
            if threshold:
                r = np.where(r > threshold, r, 0).astype(X.dtype)
            nr, nc = np.nonzero(r)
            rows.append(nr)
            cols.append(nc + js)
            vals.append(r[nr, nc])
        rows = np.concatenate(rows)
        cols = np.concatenate(cols)
        vals = np.concatenate(vals)
        order = np.lexsort((cols, rows))
        blk = ((rows[order].astype(np.int32), cols[order].astype(np.int32)), vals[order])
        if update_normalization:
            return blk, c
        return blk

    def _rebalance(self, X, bi, new_c):
        """Rescale, renormalise, and fold the drift into c (lakde/local_adaptive_kde.py:156-181)."""
        N = len(X)
        fi = np.finfo(X.dtype)
        with np.errstate(over="ignore", invalid="ignore"):
            coeff = np.clip(np.exp(self.rnm_log_consts - new_c), fi.tiny, fi.max).astype(X.dtype)
        sums = np.zeros(N, dtype=X.dtype)
        for bj in range(len(self.rnm_blocks)):
            (row, col), val = self.rnm_blocks[bj]
            col = col.astype(np.int64)
            if bj != bi:
                val = (val * coeff[col]).astype(X.dtype)
                self.rnm_blocks[bj] = ((row, col.astype(np.int32)), val)
            np.add.at(sums, col, val)
        sums = np.maximum(sums, fi.eps).astype(X.dtype)
        new_c = (new_c + np.log(sums)).astype(X.dtype)
        coeff = np.clip((1 / sums).astype(X.dtype), fi.tiny, fi.max).astype(X.dtype)
        for bj in range(len(self.rnm_blocks)):
            (row, col), val = self.rnm_blocks[bj]
            self.rnm_blocks[bj] = ((row, col), (val * coeff[col.astype(np.int64)]).astype(X.dtype))
        return new_c

    def _init_common(self, X, threshold, include_self):
        N, D = X.shape
        dt = X.dtype
        self.dtype = dt
        self.eps = np.finfo(dt).eps
        self.block_size = min(self.block_size, N)
        self.W_inv_jitter = np.zeros(N, dtype=dt)
        self.a_0 = np.asarray(self.a_0_arg, dtype=dt)
        self.b_0 = np.asarray(self.b_0_arg, dtype=dt)
        self.nu_0 = np.asarray(D if self.nu_0_arg is None else self.nu_0_arg, dtype=dt)
        if self.nu_0 <= D - 1:
            raise ValueError("nu_0 must be greater than the data dimensionality minus one")
        if isinstance(self.k_arg, int):
            self.knn_graph = knn_graph(X, self.k_arg, include_self=include_self)
        else:
            self.knn_graph = np.asarray(self.k_arg)
        self.k = self.knn_graph.shape[1]
        if threshold:
            init_k = min(math.floor(1 / threshold), self.k)
        else:
            init_k = self.k
        inds = knn_pattern(self.knn_graph[:, :init_k], self.block_size)
        self.rnm_blocks = [
            ((ix[0].astype(np.int32), ix[1].astype(np.int32)), np.full(ix.shape[1], 1 / init_k, dtype=dt))
            for ix in inds
        ]
        self.nu = np.empty(N, dtype=dt)
        self.a = np.full(N, self.a_0 + self.nu_0 * D / 2, dtype=dt)
        self.b = self.a.copy()
        self.rnm_log_consts = np.full(N, -np.inf, dtype=dt)
        self.logdet_W = np.empty(N, dtype=dt)

    def _dense_normaliser_pass(self, X, bi, W_triu, nu):
        N = len(X)
        s, e = self._blocks(N)[bi]
        logdet_W = chol_logdet(W_triu)
        for bj, (js, je) in enumerate(self._blocks(N)):
            log_rho = calc_log_rho_block(X[js:je], X[s:e], nu, W_triu, logdet_W)
            log_rho = self._mask_block(log_rho, bi, bj, N)
            self.rnm_log_consts[js:je] = np.logaddexp(self.rnm_log_consts[js:je], logsumexp0(log_rho))

    def fit(self, X, iterations=10, threshold=None, callback=None):
        X = np.ascontiguousarray(X)
        if not threshold:
            threshold = 0
        if self.iter_steps < 1:
            self.init_parameters_(X, threshold)
            self.init_summaries_(X, threshold)
        nb = len(self._blocks(len(X)))
        for _ in range(iterations):
            for bi in range(nb):
                self.partial_step_(X, bi, threshold)
                if callback is not None:
                    callback(self, X)
                self.iter_steps += 1
        return self

    def data_log_likelihood_no_rnm(self, X):
        D = X.shape[1]
        return (-D / 2 * math.log(2 * math.pi) + self.rnm_log_consts).astype(X.dtype)

    def log_pred_density(self, X, Y):
        """Student-t mixture predictive density (lakde/local_adaptive_kde.py:200-223)."""
        N, D = X.shape
        out = np.full(len(Y), -np.inf, dtype=X.dtype)
        for bi, (s, e) in enumerate(self._blocks(N)):
            S, nu = self._posterior_contribs(X, bi)
            sigma_0 = self.prior_cov(X, bi)[0]
            W_triu = self._posterior(bi, N, sigma_0, S)
            log_coeff = (
                lgamma((nu + 1) / 2).astype(np.float64)
                - lgamma((nu + 1 - D) / 2).astype(np.float64)
                + 0.5 * chol_logdet(W_triu)
                - D / 2 * LOGPI
            ).astype(X.dtype)
            for js in range(0, len(Y), self.block_size):
                Q = chol_quad_form(W_triu, X[s:e], Y[js : js + self.block_size])
                lp = log_coeff[:, None] - (nu[:, None] + 1) / 2 * np.log1p(Q)
                out[js : js + self.block_size] = np.logaddexp(
                    out[js : js + self.block_size], logsumexp0(lp.astype(X.dtype))
                )
        return (-math.log(N) + out).astype(X.dtype)

    def posterior_factors(self, X):
        """(W_triu, nu, logdet_W) recomputed from the current r, as log_pred_density does."""
        N = len(X)
        Ws, nus = [], []
        for bi in range(len(self._blocks(N))):
            S, nu = self._posterior_contribs(X, bi)
            sigma_0 = self.prior_cov(X, bi)[0]
            Ws.append(self._posterior(bi, N, sigma_0, S))
            nus.append(nu)
        W = np.concatenate(Ws)
        return W, np.concatenate(nus), chol_logdet(W)


def expect_log_p_tau(a_0, b_0, e_tau, e_log_tau):
    """lakde/local_adaptive_kde.py:21-26."""
    return np.sum(-lgamma(a_0) + a_0 * np.log(b_0) + (a_0 - 1) * e_log_tau - b_0 * e_tau)


def expect_log_q_tau(a, b, e_tau, e_log_tau):
    """lakde/local_adaptive_kde.py:29-33."""
    return np.sum(-lgamma(a) + a * np.log(b) + (a - 1) * e_log_tau - b * e_tau)


class KNNKDEOracle(_AdaptiveOracle):
    """LocalKNearestKDE (lakde/local_knn_kde.py:50-341)."""

    def init_parameters_(self, X, threshold):
        """lakde/local_knn_kde.py:73-138."""
        self._init_common(X, threshold, include_self=False)
        N = len(X)
        self.sigma_0_jitter = np.zeros(N, dtype=X.dtype)
        self.logdet_sigma_0 = np.empty(N, dtype=X.dtype)
        self.sigma_0_lambda_mm_trace = np.empty(N, dtype=X.dtype)

    def prior_cov(self, X, bi):
        """Sigma0 from the kNN covariance + its jittered Cholesky (lakde/local_knn_kde.py:195-207)."""
        s, e = self._blocks(len(X))[bi]
        sigma_0 = batched_knn_cov(X, X[s:e], self.knn_graph[s:e].astype(np.int64))
        L, jit = stabilized_cholesky(sigma_0, self.sigma_0_jitter[s:e], eps=self.eps)
        if jit is not None:
            self.sigma_0_jitter[s:e] = jit
        sigma_0 = _with_jitter(sigma_0, self.sigma_0_jitter[s:e])
        return sigma_0, L

    def init_summaries_(self, X, threshold):
        """lakde/local_knn_kde.py:140-193."""
        N = len(X)
        for bi, (s, e) in enumerate(self._blocks(N)):
            sigma_0, sigma_0_tril = self.prior_cov(X, bi)
            S, nu = self._posterior_contribs(X, bi)
            W_triu = self._posterior(bi, N, sigma_0, S)
            self.nu[s:e] = nu
            self.logdet_W[s:e] = chol_logdet(W_triu)
            self.logdet_sigma_0[s:e] = chol_logdet(sigma_0_tril)
            self.sigma_0_lambda_mm_trace[s:e] = nu * chol_mm_trace(sigma_0_tril, W_triu)
            self._dense_normaliser_pass(X, bi, W_triu, nu)
        for bi in range(len(self._blocks(N))):
            sigma_0, _ = self.prior_cov(X, bi)
            S, nu = self._posterior_contribs(X, bi)
            W_triu = self._posterior(bi, N, sigma_0, S)
            self.rnm_blocks[bi] = self._expectation(X, bi, W_triu, nu, False, threshold)
        self.rnm_log_consts = self._rebalance(X, -1, self.rnm_log_consts)

    def partial_step_(self, X, bi, threshold):
        """lakde/local_knn_kde.py:209-254."""
        N = len(X)
        s, e = self._blocks(N)[bi]
        sigma_0, sigma_0_tril = self.prior_cov(X, bi)
        S, nu = self._posterior_contribs(X, bi)
        W_triu = self._posterior(bi, N, sigma_0, S)
        blk, new_c = self._expectation(X, bi, W_triu, nu, True, threshold)
        mm = nu * chol_mm_trace(sigma_0_tril, W_triu)
        self.rnm_blocks[bi] = blk
        self.logdet_W[s:e] = chol_logdet(W_triu)
        self.logdet_sigma_0[s:e] = chol_logdet(sigma_0_tril)
        self.sigma_0_lambda_mm_trace[s:e] = mm
        self.nu[s:e] = nu
        self.b[s:e] = self.b_0 + self.nu_0 * mm / 2
        self.rnm_log_consts = self._rebalance(X, bi, new_c)

    def compute_elbo(self, X):
        """lakde/local_knn_kde.py:256-341 with the terms of :24-47."""
        N, D = X.shape
        nu_0 = self.nu_0
        e_tau = self.a / self.b
        e_log_tau = scipy.special.digamma(self.a.astype(np.float64)).astype(X.dtype) - np.log(self.b)
        e_logdet = mvdigamma(self.nu / 2, D) + D * LOG2 + self.logdet_W
        p_tau = expect_log_p_tau(self.a_0, self.b_0, e_tau, e_log_tau)
        q_tau = expect_log_q_tau(self.a, self.b, e_tau, e_log_tau)
        B_p = -nu_0 / 2 * (D * LOG2 - self.logdet_sigma_0 - D * e_log_tau - D * np.log(nu_0)) - mvlgamma(nu_0 / 2, D)
        p_lam = np.sum(B_p + (nu_0 - D - 1) * e_logdet / 2 - e_tau * nu_0 * self.sigma_0_lambda_mm_trace / 2)
        B_q = -self.nu / 2 * (self.logdet_W + D * LOG2) - mvlgamma(self.nu / 2, D)
        q_lam = np.sum(B_q + (self.nu - D - 1) * e_logdet / 2 - self.nu / 2 * D)
        log_z_p = -N * math.log(N - 1)
        ll = self.data_log_likelihood_no_rnm(X).sum()
        return float(ll + (p_lam - q_lam) + log_z_p + (p_tau - q_tau))


class HierKDEOracle(_AdaptiveOracle):
    """LocalHierarchicalKDE (lakde/local_hierarchical_kde.py:82-461)."""

    def __init__(self, nu_0=None, k=20, block_size=512, nu_shared_0=None, a_0=1e-6, b_0=1e-6, candidates=None):
        super().__init__(nu_0, k, block_size, a_0, b_0, candidates)
        self.nu_shared_0_arg = nu_shared_0

    def init_parameters_(self, X, threshold):
        """lakde/local_hierarchical_kde.py:111-196."""
        N, D = X.shape
        self._init_common(X, threshold, include_self=True)
        self.W_shared_inv_jitter = np.zeros((), dtype=X.dtype)
        self.nu_shared_0 = np.asarray(
            D - 1 + 1e-2 if self.nu_shared_0_arg is None else self.nu_shared_0_arg, dtype=X.dtype
        )
        if self.nu_shared_0 <= D - 1:
            raise ValueError("nu_shared_0 must be greater than the data dimensionality minus one")
        sigma_0 = cov(X)
        sigma_0_tril, _ = stabilized_cholesky(sigma_0)
        self.lambda_0_triu = tril_inverse(sigma_0_tril).T
        self.lambda_0 = self.lambda_0_triu @ self.lambda_0_triu.T
        self.nu_shared = float(self.nu_shared_0) + N * float(self.nu_0)
        self.W_shared_triu = float(self.nu_0) * sigma_0_tril.T / self.nu_shared
        self.expect_lambda_contribs = np.empty((len(self._blocks(N)), D, D), dtype=np.float64)

    def prior_cov(self, X=None, bi=None):
        """Shared E[Sigma_bar] and its triangular factor (lakde/local_hierarchical_kde.py:269-271)."""
        triu = math.sqrt(self.nu_shared) * self.W_shared_triu
        return triu @ triu.T, triu

    def _lambda_contrib(self, W_triu, nu, e_tau):
        c = (W_triu @ np.swapaxes(W_triu, -1, -2)) * (nu * e_tau)[:, None, None]
        return c.astype(W_triu.dtype).astype(np.float64).sum(0)

    def init_summaries_(self, X, threshold):
        """lakde/local_hierarchical_kde.py:198-258."""
        N = len(X)
        sigma_bar, _ = self.prior_cov()
        for bi, (s, e) in enumerate(self._blocks(N)):
            S, nu = self._posterior_contribs(X, bi)
            W_triu = self._posterior(bi, N, sigma_bar, S)
            self.nu[s:e] = nu
            self.logdet_W[s:e] = chol_logdet(W_triu)
            e_tau = self.a[s:e] / self.b[s:e]
            self.expect_lambda_contribs[bi] = self._lambda_contrib(W_triu, nu, e_tau)
            self._dense_normaliser_pass(X, bi, W_triu, nu)
        for bi in range(len(self._blocks(N))):
            S, nu = self._posterior_contribs(X, bi)
            W_triu = self._posterior(bi, N, sigma_bar, S)
            self.rnm_blocks[bi] = self._expectation(X, bi, W_triu, nu, False, threshold)
        self.rnm_log_consts = self._rebalance(X, -1, self.rnm_log_consts)

    def partial_step_(self, X, bi, threshold):
        """lakde/local_hierarchical_kde.py:273-332.

        Note: the trace term uses chol_mm_trace(E[Sigma_bar], W_triu), i.e. the
        full matrix E[Sigma_bar] in the place of a triangular factor, exactly as
        the reference does at lakde/local_hierarchical_kde.py:286-288.
        """
        N = len(X)
        s, e = self._blocks(N)[bi]
        sigma_bar, _ = self.prior_cov()
        S, nu = self._posterior_contribs(X, bi)
        W_triu = self._posterior(bi, N, sigma_bar, S)
        blk, new_c = self._expectation(X, bi, W_triu, nu, True, threshold)
        mm = nu * chol_mm_trace(sigma_bar.astype(W_triu.dtype), W_triu)
        b = (self.b_0 + self.nu_0 * mm / 2).astype(X.dtype)
        e_tau = self.a[s:e] / b
        contrib = self._lambda_contrib(W_triu, nu, e_tau)
        self.rnm_blocks[bi] = blk
        self.expect_lambda_contribs[bi] = contrib
        prec = self.expect_lambda_contribs.sum(0) * float(self.nu_0) + float(self.nu_shared_0) * self.lambda_0
        jit = self.W_shared_inv_jitter
        L, jit = stabilized_cholesky(prec, jit, eps=np.finfo(np.float64).eps)
        if jit is not None:
            self.W_shared_inv_jitter = jit
        self.W_shared_triu = tril_inverse(L).T
        self.logdet_W[s:e] = chol_logdet(W_triu)
        self.nu[s:e] = nu
        self.b[s:e] = b
        self.rnm_log_consts = self._rebalance(X, bi, new_c)

    def compute_elbo(self, X):
        """lakde/local_hierarchical_kde.py:334-461 with the terms of :25-79."""
        N, D = X.shape
        nu_0 = self.nu_0
        e_tau = self.a / self.b
        triu = math.sqrt(self.nu_shared) * self.W_shared_triu
        sigma_bar = triu @ triu.T
        e_log_tau = scipy.special.digamma(self.a.astype(np.float64)).astype(X.dtype) - np.log(self.b)
        e_logdet = mvdigamma(self.nu / 2, D) + D * LOG2 + self.logdet_W
        lam_sum = self.expect_lambda_contribs.sum(0)
        logdet_sigma_0 = -chol_logdet(self.lambda_0_triu)
        logdet_W_shared = np.asarray(chol_logdet(self.W_shared_triu), dtype=X.dtype)
        nu_sh = np.asarray(self.nu_shared, dtype=np.float64)
        e_logdet_sh = mvdigamma(nu_sh / 2, D) + D * LOG2 + logdet_W_shared
        tr_lam = np.trace(sigma_bar @ lam_sum)
        tr_lam0 = np.trace(sigma_bar @ self.lambda_0)
        p_tau = expect_log_p_tau(self.a_0, self.b_0, e_tau, e_log_tau)
        q_tau = expect_log_q_tau(self.a, self.b, e_tau, e_log_tau)
        B_p = -nu_0 / 2 * (D * LOG2 - D * e_log_tau - D * np.log(nu_0) - e_logdet_sh) - mvlgamma(nu_0 / 2, D)
        p_lam = np.sum(B_p + (nu_0 - D - 1) * e_logdet / 2) - nu_0 * tr_lam / 2
        B_q = -self.nu / 2 * (self.logdet_W + D * LOG2) - mvlgamma(self.nu / 2, D)
        q_lam = np.sum(B_q + (self.nu - D - 1) * e_logdet / 2 - self.nu * D / 2)
        nsh0 = self.nu_shared_0
        p_sh = (
            -nsh0 / 2 * (logdet_sigma_0 + D * LOG2 - D * np.log(nsh0))
            - mvlgamma(nsh0 / 2, D)
            + (nsh0 - D - 1) * e_logdet_sh / 2
            - nsh0 * tr_lam0 / 2
        )
        q_sh = (
            -nu_sh / 2 * (logdet_W_shared + D * LOG2)
            - mvlgamma(nu_sh / 2, D)
            + (nu_sh - D - 1) * e_logdet_sh / 2
            - nu_sh * D / 2
        )
        log_z_p = -N * math.log(N - 1)
        ll = self.data_log_likelihood_no_rnm(X).sum()
        return float(ll + (p_lam - q_lam) + log_z_p + (p_tau - q_tau) + (p_sh - q_sh))


# ---------------------------------------------------------------------------
# functional predictive density (for gradient checks)
# ---------------------------------------------------------------------------


def log_pred_density_from_factors(X, Y, W_triu, nu, logdet_W):
    """log p(y) = -log N + logsumexp_n[log_coeff_n - (nu_n+1)/2 log1p(Q_ny)].

    The formula of lakde/local_adaptive_kde.py:209-223 as a pure function of the
    posterior factors, evaluated in the dtype of the inputs.
    """
    N, D = X.shape
    log_coeff = (
        lgamma((nu + 1) / 2).astype(np.float64)
        - lgamma((nu + 1 - D) / 2).astype(np.float64)
        + 0.5 * logdet_W
        - D / 2 * LOGPI
    ).astype(X.dtype)
    Q = chol_quad_form(W_triu, X, Y)
    lp = log_coeff[:, None] - (nu[:, None] + 1) / 2 * np.log1p(Q)
    return (-math.log(N) + logsumexp0(lp.astype(X.dtype))).astype(X.dtype)


# ---------------------------------------------------------------------------
# the E-step on a fixed pair pattern at block_size = N
# (lakde/local_adaptive_kde.py:98-181 with pairs outside the pattern at -inf)
# ---------------------------------------------------------------------------


def sparse_log_rho(rowptr, col, X, W_triu, nu, logdet_W, kernel_offset=0):
    """log rho for the pairs of a kernel-major CSR pattern (lakde/local_adaptive_kde.py:36-44, 126-128)."""
    rows = _rows_of(rowptr)
    col = np.asarray(col, dtype=np.int64)
    D = X.shape[1]
    self_idx = rows + kernel_offset
    delta = X[col] - X[self_idx]
    y = np.einsum("pji,pj->pi", np.triu(W_triu)[rows], delta, optimize=True)
    Q = (y * y).sum(-1)
    lr = (Q * (-0.5 * nu[rows]) + log_rho_const(nu, logdet_W, D)[rows]).astype(X.dtype)
    lr[col == self_idx] = -np.inf
    return lr


def sparse_normalise(col, logrho, c, rsum, npts, mode, threshold=0.0):
    """Per-point normaliser, thresholded responsibilities and rebalance.

    mode 0 restates the initial pass (lakde/local_knn_kde.py:157-193:
    c = logaddexp(c, logsumexp), then r and the rebalance); mode 1 the update
    (lakde/local_adaptive_kde.py:120-145 at block_size = N, then :156-181).
    Returns (r, c_new, rsum_new).
    """
    dt = logrho.dtype
    col = np.asarray(col, dtype=np.int64)
    fi = np.finfo(dt)
    mx = np.full(npts, -np.inf, dtype=dt)
    np.maximum.at(mx, col, logrho)
    ms = np.where(np.isfinite(mx), mx, 0).astype(dt)
    se = np.zeros(npts, dtype=dt)
    with np.errstate(invalid="ignore"):
        np.add.at(se, col, np.exp(logrho - ms[col]).astype(dt))
    with np.errstate(divide="ignore"):
        lse = np.where(np.isfinite(mx), np.log(se) + ms, -np.inf).astype(dt)
    if mode == 0:
        c_new = np.logaddexp(c, lse).astype(dt)
    else:
        with np.errstate(divide="ignore"):
            old = (np.log(rsum) + c).astype(dt)
        c_new = np.logaddexp(logsubexp(c, old), lse).astype(dt)
    with np.errstate(invalid="ignore"):
        r = np.exp(logrho - c_new[col]).astype(dt)
    if threshold:
        r = np.where(r > threshold, r, 0).astype(dt)
    sums = np.zeros(npts, dtype=dt)
    np.add.at(sums, col, r)
    sums = np.maximum(sums, fi.eps).astype(dt)
    c_fin = (c_new + np.log(sums)).astype(dt)
    coeff = np.clip((1 / sums).astype(dt), fi.tiny, fi.max).astype(dt)
    r = (r * coeff[col]).astype(dt)
    rs = np.zeros(npts, dtype=dt)
    np.add.at(rs, col, r)
    return r, c_fin, rs
