"""LocalHierarchicalKDE: per-kernel Wishart posteriors with a learned shared
prior (lakde/local_hierarchical_kde.py)."""

import math
from typing import Union

import numpy as np
import torch

from . import kernels as K
from .engine import FusedHier, build_pattern
from .linalg_util import chol_logdet, chol_mm_trace, mvdigamma, mvlgamma, stabilized_cholesky, tril_inverse
from .local_adaptive_kde import (
    LocallyAdaptiveKDE,
    calc_log_rho_block,
    expect_log_p_tau,
    expect_log_q_tau,
)
from .sparse_util import graph_to_slices
from .utils import InterruptDelay, compute_knn_graph, cov, tensor_as


class LocalHierarchicalKDE(LocallyAdaptiveKDE):
    """Same constructor, fit() and log_pred_density() as lakde.LocalHierarchicalKDE,
    plus the ``fused`` / ``candidates`` / ``cuda_graph`` options of LocalKNearestKDE."""

    def __init__(self, nu_0: Union[torch.Tensor, float] = None, k_or_knn_graph: Union[torch.Tensor, int] = None,
                 block_size: int = 512, nu_shared_0: Union[torch.Tensor, float] = None,
                 a_0: Union[torch.Tensor, float] = 1e-6, b_0: Union[torch.Tensor, float] = 1e-6, verbose=False,
                 logs=False, fused=False, candidates="knn", cuda_graph=True, candidate_counts=None,
                 precision="auto", autotune=True):
        super().__init__(nu_0, a_0, b_0, block_size, verbose, logs, fused, candidates, cuda_graph)
        self.autotune = autotune
        self.k_or_knn_graph = k_or_knn_graph
        self.candidate_counts = candidate_counts
        self.precision = precision
        self.knn_graph = None
        self.k = None
        self.nu_shared_0 = nu_shared_0
        self.lambda_0_triu = None
        self.lambda_0 = None
        self.nu_shared = None
        self.W_shared_triu = None
        self.expect_lambda_contribs = None
        self.W_shared_inv_jitter = None

    def init_parameters_(self, X, sparsity_threshold=None):
        """lakde/local_hierarchical_kde.py:111-196."""
        N, D = X.shape
        self.block_size = N if self.fused else min(self.block_size, N)
        self.a_0 = tensor_as(self.a_0, X)
        self.b_0 = tensor_as(self.b_0, X)
        self.nu_0 = tensor_as(self.nu_0, X) if self.nu_0 is not None else X.new_full((), D)
        if bool(torch.any(self.nu_0 <= D - 1)):
            raise ValueError(
                "nu_0 must be greater than the data dimensionality minus one, or the ELBO will be undefined"
            )
        self.nu_shared_0 = (tensor_as(self.nu_shared_0, X) if self.nu_shared_0 is not None
                            else X.new_full((), D - 1 + 1e-2))
        if float(self.nu_shared_0) <= D - 1:
            raise ValueError(
                "nu_shared_0 must be greater than the data dimensionality minus one, or the ELBO will be undefined"
            )
        g = self.k_or_knn_graph
        if isinstance(g, int):
            if self.verbose:
                print("Computing nearest neighbour graph...")
            self.knn_graph = compute_knn_graph(X, g, 1024, include_self=True, metric="l2", dtype=torch.int32)
        elif isinstance(g, np.ndarray):
            self.knn_graph = torch.from_numpy(g).to(X.device)
        elif torch.is_tensor(g) and g.dtype in (torch.int32, torch.int64):
            self.knn_graph = g.to(X.device)
        else:
            raise ValueError("k_or_knn_graph type not recognised")
        self.k = self.knn_graph.size(-1)
        init_k = min(math.floor(1 / sparsity_threshold), self.k) if sparsity_threshold else self.k
        if self.fused:
            pattern = build_pattern(self.candidates, self.knn_graph, N, X.device, self.candidate_counts)
            self.engine = FusedHier(X, self.knn_graph, pattern, self.nu_0, self.a_0, self.b_0, sparsity_threshold,
                                    init_k, self.nu_shared_0, self.precision)
            self._eager_steps = 0
            self._sync_from_engine()
            self._sync_shared()
            return
        self.W_shared_inv_jitter = torch.zeros((), dtype=torch.float64, device=X.device)
        self.W_inv_jitter = X.new_zeros(N)
        sigma_0 = cov(X, dtype=torch.double)
        sigma_0_tril, _ = stabilized_cholesky(sigma_0)
        self.lambda_0_triu = tril_inverse(sigma_0_tril).T
        self.lambda_0 = self.lambda_0_triu @ self.lambda_0_triu.T
        inds = graph_to_slices(self.knn_graph[:, :init_k], self.block_size)
        self.knn_graph = None  # only needed for the initial pattern
        self.rnm_blocks = [(ix.to(torch.int32), X.new_full((ix.size(1),), 1 / init_k)) for ix in inds]
        self.nu_shared = self.nu_shared_0 + N * self.nu_0.double()
        self.W_shared_triu = self.nu_0 * sigma_0_tril.T / self.nu_shared
        self.nu = X.new_empty(N)
        self.a = (self.a_0 + self.nu_0 * D / 2).expand(N).contiguous()
        self.b = self.a.clone()
        self.rnm_active_contribs = X.new_zeros(())
        self.rnm_log_consts = X.new_full((N,), -math.inf)
        self.logdet_W = X.new_empty(N)
        self.expect_lambda_contribs = X.new_empty(self.num_blocks(N), D, D, dtype=torch.double)

    def resume_(self, X, sparsity_threshold=None):
        """Continues from a restored state dict.  The fused engine is rebuilt:
        the candidate pattern from the kNN graph of ``k_or_knn_graph``
        (recomputed from X when it is a count), then r, c, the per-kernel state
        and the shared precision from the checkpoint."""
        N, D = X.shape
        self._resume_tensors(X, self._STATE_KEYS + self._HIER_KEYS)
        if not self.fused or self.engine is not None:
            return
        self.a_0 = tensor_as(self.a_0, X)
        self.b_0 = tensor_as(self.b_0, X)
        self.nu_0 = tensor_as(self.nu_0, X)
        g = self.k_or_knn_graph
        if isinstance(g, int):
            graph = compute_knn_graph(X, g, 1024, include_self=True, metric="l2", dtype=torch.int32)
        else:
            graph = (torch.from_numpy(g) if isinstance(g, np.ndarray) else g).to(X.device)
        self.k = graph.size(-1)
        init_k = min(math.floor(1 / sparsity_threshold), self.k) if sparsity_threshold else self.k
        pattern = build_pattern(self.candidates, graph, N, X.device, self.candidate_counts)
        eng = FusedHier(X, graph, pattern, self.nu_0, self.a_0, self.b_0, sparsity_threshold, init_k,
                        tensor_as(self.nu_shared_0, X), self.precision)
        self._restore_engine_state(eng)
        eng.W_shared_triu.copy_(self.W_shared_triu.to(eng.W_shared_triu.dtype))
        eng.expect_lambda_contribs[0] = self.expect_lambda_contribs.sum(0)
        eng.W_shared_inv_jitter.copy_(self.W_shared_inv_jitter.reshape(-1)[:1].to(torch.float64))
        eng._refresh_prior()
        self.engine = eng
        self._eager_steps = 0
        self._sync_from_engine()
        self._sync_shared()
        self.block_size = N

    def _sync_shared(self):
        eng = self.engine
        self.lambda_0_triu = eng.lambda_0_triu
        self.lambda_0 = eng.lambda_0
        self.nu_shared = torch.tensor(eng.nu_shared, dtype=torch.float64, device=eng.device)
        self.W_shared_triu = eng.W_shared_triu
        self.expect_lambda_contribs = eng.expect_lambda_contribs
        self.W_shared_inv_jitter = eng.W_shared_inv_jitter

    def _expect_lambda_contrib(self, W_triu, nu, e_tau):
        c = W_triu @ W_triu.mT
        c *= (nu * e_tau)[:, None, None]
        return torch.sum(c, dtype=torch.double, dim=0)

    def init_summaries_(self, X, sparsity_threshold=None):
        """lakde/local_hierarchical_kde.py:198-258."""
        if self.fused:
            self.engine.init_summaries()
            self._sync_from_engine()
            self._sync_shared()
            return
        N = X.size(0)
        sigma_bar, _ = self.calc_prior_cov()
        for bi, i in enumerate(range(0, N, self.block_size)):
            X_train = X[i : i + self.block_size]
            S, nu = self.calc_posterior_contribs(X, bi)
            W_triu = self.calc_posterior(bi, sigma_bar, S)
            logdet_W = chol_logdet(W_triu)
            sl = slice(i, i + self.block_size)
            self.nu[sl] = nu
            self.logdet_W[sl] = logdet_W
            self.expect_lambda_contribs[bi] = self._expect_lambda_contrib(W_triu, nu, self.a[sl] / self.b[sl])
            for bj, j in enumerate(range(0, N, self.block_size)):
                log_rho = calc_log_rho_block(X[j : j + self.block_size], X_train, nu, W_triu, logdet_W)
                if bi == bj:
                    log_rho.diagonal().fill_(-math.inf)
                jl = slice(j, j + self.block_size)
                torch.logaddexp(self.rnm_log_consts[jl], torch.logsumexp(log_rho, dim=0), out=self.rnm_log_consts[jl])
        for bi in range(self.num_blocks(N)):
            S, nu = self.calc_posterior_contribs(X, bi)
            W_triu = self.calc_posterior(bi, sigma_bar, S)
            self.rnm_blocks[bi] = self.partial_expectation_step(X, bi, W_triu, nu, update_normalization=False,
                                                                sparsity_threshold=sparsity_threshold)
            self.rnm_active_contribs += self.rnm_blocks[bi][1].numel()
        self.rnm_log_consts = self.rebalance_responsibilities_(X, -1, self.rnm_log_consts)

    def calc_prior_prec(self):
        """lakde/local_hierarchical_kde.py:260-267."""
        return self.expect_lambda_contribs.sum(dim=0).mul_(float(self.nu_0)).add_(self.lambda_0,
                                                                                   alpha=float(self.nu_shared_0))

    def calc_prior_cov(self, *_):
        """E[Sigma_bar] and its triangular factor (lakde/local_hierarchical_kde.py:269-271)."""
        triu = torch.sqrt(self.nu_shared) * self.W_shared_triu
        return triu @ triu.T, triu

    def partial_step_(self, X, block_idx, sparsity_threshold=None):
        """lakde/local_hierarchical_kde.py:273-332."""
        if self.fused:
            self._fused_step()
            return
        s, e = self._span(block_idx)
        sigma_bar, _ = self.calc_prior_cov()
        S, nu = self.calc_posterior_contribs(X, block_idx)
        W_triu = self.calc_posterior(block_idx, sigma_bar, S)
        indices, values, new_c = self.partial_expectation_step(X, block_idx, W_triu, nu,
                                                               sparsity_threshold=sparsity_threshold)
        logdet_W = chol_logdet(W_triu)
        # the full matrix E[Sigma_bar] in the place of a triangular factor, as
        # the reference computes it (lakde/local_hierarchical_kde.py:286-288)
        mm = nu * chol_mm_trace(sigma_bar.to(W_triu.dtype), W_triu)
        b = self.b_0 + self.nu_0 * mm / 2
        contrib = self._expect_lambda_contrib(W_triu, nu, self.a[s:e] / b)
        with InterruptDelay():
            self.rnm_active_contribs -= self.rnm_blocks[block_idx][1].numel()
            self.rnm_active_contribs += values.numel()
            self.rnm_blocks[block_idx] = (indices.to(torch.int32), values)
            self.expect_lambda_contribs[block_idx] = contrib
            W_shared_inv_tril, jit = stabilized_cholesky(self.calc_prior_prec(), self.W_shared_inv_jitter)
            if jit is not None:
                self.W_shared_inv_jitter = jit
            self.W_shared_triu = tril_inverse(W_shared_inv_tril).T
            self.logdet_W[s:e] = logdet_W
            self.nu[s:e] = nu
            self.b[s:e] = b
            self.rnm_log_consts = self.rebalance_responsibilities_(X, block_idx, new_c)

    def compute_elbo(self, X):
        """lakde/local_hierarchical_kde.py:334-461 (FP64 reductions on the fused path)."""
        if self.fused:
            return self.engine.compute_elbo()
        N, D = X.shape
        expect_tau = self.a / self.b
        triu = torch.sqrt(self.nu_shared) * self.W_shared_triu
        sigma_bar = triu @ triu.T
        e_log_tau = torch.digamma(self.a) - torch.log(self.b)
        e_logdet = mvdigamma(self.nu / 2, D) + D * math.log(2) + self.logdet_W
        lam_sum = self.expect_lambda_contribs.sum(dim=0)
        logdet_sigma_0 = -chol_logdet(self.lambda_0_triu)
        logdet_W_shared = chol_logdet(self.W_shared_triu).to(X.dtype)
        e_logdet_sh = mvdigamma(self.nu_shared / 2, D) + D * math.log(2) + logdet_W_shared
        tr_lam = torch.trace(sigma_bar @ lam_sum)
        tr_lam0 = torch.trace(sigma_bar @ self.lambda_0)
        p_tau = expect_log_p_tau(self.a_0, self.b_0, expect_tau, e_log_tau)
        q_tau = expect_log_q_tau(self.a, self.b, expect_tau, e_log_tau)
        nu_0 = self.nu_0
        B_p = -nu_0 / 2 * (D * math.log(2) - D * e_log_tau - D * torch.log(nu_0) - e_logdet_sh) - mvlgamma(nu_0 / 2, D)
        p_lam = torch.sum(B_p + (nu_0 - D - 1) * e_logdet / 2) - nu_0 * tr_lam / 2
        B_q = -self.nu / 2 * (self.logdet_W + D * math.log(2)) - mvlgamma(self.nu / 2, D)
        q_lam = torch.sum(B_q + (self.nu - D - 1) * e_logdet / 2 - self.nu * D / 2)
        nsh0, nsh = self.nu_shared_0, self.nu_shared
        p_sh = (-nsh0 / 2 * (logdet_sigma_0 + D * math.log(2) - D * torch.log(nsh0)) - mvlgamma(nsh0 / 2, D)
                + (nsh0 - D - 1) * e_logdet_sh / 2 - nsh0 * tr_lam0 / 2)
        q_sh = (-nsh / 2 * (logdet_W_shared + D * math.log(2)) - mvlgamma(nsh / 2, D)
                + (nsh - D - 1) * e_logdet_sh / 2 - nsh * D / 2)
        ll = self.data_log_likelihood_no_rnm(X).sum()
        return ll + (p_lam - q_lam) - N * math.log(N - 1) + (p_tau - q_tau) + (p_sh - q_sh)

    _HIER_KEYS = ("k", "nu_shared_0", "nu_shared", "lambda_0", "lambda_0_triu", "W_shared_triu",
                  "expect_lambda_contribs", "W_shared_inv_jitter")

    def state_dict(self):
        d = super().state_dict()
        d.update({k: getattr(self, k) for k in self._HIER_KEYS})
        return d

    def load_state_dict(self, state_dict):
        super().load_state_dict(state_dict)
        for k in self._HIER_KEYS:
            setattr(self, k, state_dict[k])

    def hparam_state_dict(self):
        d = super().hparam_state_dict()
        d.update({"k": self.k, "model": "hierarchical"})
        return d
