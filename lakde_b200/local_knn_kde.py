"""LocalKNearestKDE: per-kernel Wishart posteriors with a kNN-covariance prior
(lakde/local_knn_kde.py)."""

import math
from typing import Union

import numpy as np
import torch

from .engine import FusedKNN, build_pattern
from .linalg_util import chol_logdet, chol_mm_trace, mvdigamma, mvlgamma, stabilized_cholesky
from .local_adaptive_kde import (
    LocallyAdaptiveKDE,
    calc_log_rho_block,
    expect_log_p_tau,
    expect_log_q_tau,
)
from .sparse_util import graph_to_slices
from .utils import InterruptDelay, batched_knn_cov, compute_knn_graph, tensor_as


def expect_log_p_lambda(nu_0, expect_tau, expect_log_tau, expect_logdet_lambda, sigma_0_lambda_mm_trace,
                        logdet_sigma_0, D):
    """lakde/local_knn_kde.py:24-40."""
    B_p = -nu_0 / 2 * (D * math.log(2) - logdet_sigma_0 - D * expect_log_tau - D * torch.log(nu_0)) - mvlgamma(
        nu_0 / 2, D
    )
    return torch.sum(B_p + (nu_0 - D - 1) * expect_logdet_lambda / 2 - expect_tau * nu_0 * sigma_0_lambda_mm_trace / 2)


def expect_log_q_lambda(nu, expect_logdet_lambda, logdet_W, D):
    """lakde/local_knn_kde.py:43-47."""
    B_q = -nu / 2 * (logdet_W + D * math.log(2)) - mvlgamma(nu / 2, D)
    return torch.sum(B_q + (nu - D - 1) * expect_logdet_lambda / 2 - nu / 2 * D)


class LocalKNearestKDE(LocallyAdaptiveKDE):
    """Same constructor, fit() and log_pred_density() as lakde.LocalKNearestKDE.

    Extra keyword arguments: ``fused`` (batch VI on a fixed pair pattern,
    default False = the reference's block schedule), ``candidates`` (the pair
    pattern of the fused path: "knn", "dense", "lists" + ``candidate_counts``,
    or a PairPattern), ``cuda_graph`` (replay fused iterations as a CUDA
    graph), ``precision`` ("auto", "mixed" or "fp32") and ``autotune`` (time
    the library's launch choices on the first fused iteration and keep the
    fastest; lakde_b200.tuning).
    """

    def __init__(self, nu_0: Union[torch.Tensor, float] = None, k_or_knn_graph: Union[torch.Tensor, int] = None,
                 block_size: int = 512, a_0: Union[torch.Tensor, float] = 1e-6, b_0: Union[torch.Tensor, float] = 1e-6,
                 verbose=False, logs=False, fused=False, candidates="knn", cuda_graph=True, candidate_counts=None,
                 precision="auto", autotune=True):
        super().__init__(nu_0, a_0, b_0, block_size, verbose, logs, fused, candidates, cuda_graph)
        self.autotune = autotune
        self.k_or_knn_graph = k_or_knn_graph
        self.candidate_counts = candidate_counts
        self.precision = precision
        self.k = None
        self.knn_graph = None
        self.logdet_sigma_0 = None
        self.sigma_0_lambda_mm_trace = None
        self.sigma_0_jitter = None

    def init_parameters_(self, X, sparsity_threshold=None):
        """lakde/local_knn_kde.py:73-138."""
        N, D = X.shape
        self.block_size = N if self.fused else min(self.block_size, N)
        self.a_0 = tensor_as(self.a_0, X)
        self.b_0 = tensor_as(self.b_0, X)
        self.nu_0 = tensor_as(self.nu_0, X) if self.nu_0 is not None else X.new_full((), D)
        if float(self.nu_0) <= D - 1:
            raise ValueError(
                "nu_0 must be greater than the data dimensionality minus one, or the ELBO will be undefined"
            )
        g = self.k_or_knn_graph
        if isinstance(g, int):
            if self.verbose:
                print("Computing nearest neighbour graph...")
            self.knn_graph = compute_knn_graph(X, g, 1024, include_self=False, metric="l2", dtype=torch.int32)
        elif isinstance(g, np.ndarray):
            self.knn_graph = torch.from_numpy(g).to(X.device)
        elif torch.is_tensor(g) and g.dtype in (torch.int32, torch.int64):
            self.knn_graph = g.to(X.device)
        else:
            raise ValueError("k_or_knn_graph type not recognised")
        self.k = self.knn_graph.size(-1)
        init_k = min(math.floor(1 / sparsity_threshold), self.k) if sparsity_threshold else self.k
        self._init_k = init_k
        if self.fused:
            pattern = build_pattern(self.candidates, self.knn_graph, N, X.device, self.candidate_counts)
            self.engine = FusedKNN(X, self.knn_graph, pattern, self.nu_0, self.a_0, self.b_0, sparsity_threshold,
                                   init_k, self.precision)
            self._eager_steps = 0
            self._sync_from_engine()
            self.sigma_0_jitter = self.engine.sigma_0_jitter
            return
        self.sigma_0_jitter = X.new_zeros(N)
        self.W_inv_jitter = X.new_zeros(N)
        inds = graph_to_slices(self.knn_graph[:, :init_k], self.block_size)
        self.rnm_blocks = [(ix.to(torch.int32), X.new_full((ix.size(1),), 1 / init_k)) for ix in inds]
        self.nu = X.new_empty(N)
        self.a = (self.a_0 + self.nu_0 * D / 2).expand(N).contiguous()
        self.b = self.a.clone()
        self.rnm_active_contribs = X.new_zeros(())
        self.rnm_log_consts = X.new_full((N,), -math.inf)
        self.logdet_sigma_0 = X.new_empty(N)
        self.logdet_W = X.new_empty(N)
        self.sigma_0_lambda_mm_trace = X.new_empty(N)

    def resume_(self, X, sparsity_threshold=None):
        """Continues from a restored state dict (lakde/kdes.py:42-48 skips the
        initialisation once iter_steps > 0).  The fused engine is rebuilt: the
        candidate pattern from the saved kNN graph, the prior recomputed from X
        (deterministic), then r, c and the per-kernel state from the checkpoint."""
        N, D = X.shape
        self._resume_tensors(X, self._STATE_KEYS + self._KNN_KEYS)
        if not self.fused or self.engine is not None:
            return
        self.a_0 = tensor_as(self.a_0, X)
        self.b_0 = tensor_as(self.b_0, X)
        self.nu_0 = tensor_as(self.nu_0, X)
        self.knn_graph = self.knn_graph.to(X.device)
        self.k = self.knn_graph.size(-1)
        init_k = min(math.floor(1 / sparsity_threshold), self.k) if sparsity_threshold else self.k
        pattern = build_pattern(self.candidates, self.knn_graph, N, X.device, self.candidate_counts)
        eng = FusedKNN(X, self.knn_graph, pattern, self.nu_0, self.a_0, self.b_0, sparsity_threshold, init_k,
                       self.precision)
        eng.init_prior()
        self._restore_engine_state(eng)
        eng.sigma_0_lambda_mm_trace.copy_(self.sigma_0_lambda_mm_trace.to(eng.dtype))
        self.engine = eng
        self._eager_steps = 0
        self._sync_from_engine()
        self.sigma_0_jitter = eng.sigma_0_jitter
        self.logdet_sigma_0 = eng.logdet_sigma_0
        self.sigma_0_lambda_mm_trace = eng.sigma_0_lambda_mm_trace
        self.block_size = N

    def init_summaries_(self, X, sparsity_threshold=None):
        """lakde/local_knn_kde.py:140-193."""
        if self.fused:
            self.engine.init_summaries()
            self._sync_from_engine()
            self.logdet_sigma_0 = self.engine.logdet_sigma_0
            self.sigma_0_lambda_mm_trace = self.engine.sigma_0_lambda_mm_trace
            return
        N = X.size(0)
        for bi, i in enumerate(range(0, N, self.block_size)):
            X_train = X[i : i + self.block_size]
            sigma_0, sigma_0_tril = self.calc_prior_cov(X, bi)
            S, nu = self.calc_posterior_contribs(X, bi)
            W_triu = self.calc_posterior(bi, sigma_0, S)
            logdet_W = chol_logdet(W_triu)
            sl = slice(i, i + self.block_size)
            self.nu[sl] = nu
            self.logdet_W[sl] = logdet_W
            self.logdet_sigma_0[sl] = chol_logdet(sigma_0_tril)
            self.sigma_0_lambda_mm_trace[sl] = nu * chol_mm_trace(sigma_0_tril, W_triu)
            for bj, j in enumerate(range(0, N, self.block_size)):
                log_rho = calc_log_rho_block(X[j : j + self.block_size], X_train, nu, W_triu, logdet_W)
                if bi == bj:
                    log_rho.diagonal().fill_(-math.inf)
                jl = slice(j, j + self.block_size)
                torch.logaddexp(self.rnm_log_consts[jl], torch.logsumexp(log_rho, dim=0), out=self.rnm_log_consts[jl])
        for bi in range(self.num_blocks(N)):
            sigma_0, _ = self.calc_prior_cov(X, bi)
            S, nu = self.calc_posterior_contribs(X, bi)
            W_triu = self.calc_posterior(bi, sigma_0, S)
            self.rnm_blocks[bi] = self.partial_expectation_step(X, bi, W_triu, nu, update_normalization=False,
                                                                sparsity_threshold=sparsity_threshold)
            self.rnm_active_contribs += self.rnm_blocks[bi][1].numel()
        self.rnm_log_consts = self.rebalance_responsibilities_(X, -1, self.rnm_log_consts)

    def calc_prior_cov(self, X, block_idx):
        """kNN covariance prior and its jittered factor (lakde/local_knn_kde.py:195-207)."""
        if self.fused:
            return self.engine.sigma_0, self.engine.sigma_0_tril
        s, e = self._span(block_idx)
        sigma_0 = batched_knn_cov(X, X[s:e], self.knn_graph[s:e].long())
        jit = self.sigma_0_jitter[s:e]
        sigma_0_tril, new_jit = stabilized_cholesky(sigma_0, jit)
        jit.copy_(new_jit)
        sigma_0.diagonal(dim1=-2, dim2=-1).add_(jit[..., None])
        return sigma_0, sigma_0_tril

    def partial_step_(self, X, block_idx, sparsity_threshold=None):
        """lakde/local_knn_kde.py:209-254."""
        if self.fused:
            self._fused_step()
            return
        s, e = self._span(block_idx)
        sigma_0, sigma_0_tril = self.calc_prior_cov(X, block_idx)
        S, nu = self.calc_posterior_contribs(X, block_idx)
        W_triu = self.calc_posterior(block_idx, sigma_0, S)
        indices, values, new_c = self.partial_expectation_step(X, block_idx, W_triu, nu,
                                                               sparsity_threshold=sparsity_threshold)
        logdet_W = chol_logdet(W_triu)
        mm = nu * chol_mm_trace(sigma_0_tril, W_triu)
        with InterruptDelay():
            self.rnm_active_contribs -= self.rnm_blocks[block_idx][1].numel()
            self.rnm_active_contribs += values.numel()
            self.rnm_blocks[block_idx] = (indices.to(self.knn_graph.dtype), values)
            self.logdet_W[s:e] = logdet_W
            self.logdet_sigma_0[s:e] = chol_logdet(sigma_0_tril)
            self.sigma_0_lambda_mm_trace[s:e] = mm
            self.nu[s:e] = nu
            self.b[s:e] = self.b_0 + self.nu_0 * mm / 2
            self.rnm_log_consts = self.rebalance_responsibilities_(X, block_idx, new_c)

    def compute_elbo(self, X):
        """lakde/local_knn_kde.py:256-341 (FP64 reductions on the fused path)."""
        if self.fused:
            return self.engine.compute_elbo()
        N, D = X.shape
        expect_tau = self.a / self.b
        expect_log_tau = torch.digamma(self.a) - torch.log(self.b)
        expect_logdet_lambda = mvdigamma(self.nu / 2, D) + D * math.log(2) + self.logdet_W
        p_tau = expect_log_p_tau(self.a_0, self.b_0, expect_tau, expect_log_tau)
        q_tau = expect_log_q_tau(self.a, self.b, expect_tau, expect_log_tau)
        p_lam = expect_log_p_lambda(self.nu_0, expect_tau, expect_log_tau, expect_logdet_lambda,
                                    self.sigma_0_lambda_mm_trace, self.logdet_sigma_0, D)
        q_lam = expect_log_q_lambda(self.nu, expect_logdet_lambda, self.logdet_W, D)
        ll = self.data_log_likelihood_no_rnm(X).sum()
        return ll + (p_lam - q_lam) - N * math.log(N - 1) + (p_tau - q_tau)

    _KNN_KEYS = ("knn_graph", "k", "logdet_sigma_0", "sigma_0_lambda_mm_trace", "sigma_0_jitter")

    def state_dict(self):
        d = super().state_dict()
        d.update({k: getattr(self, k) for k in self._KNN_KEYS})
        return d

    def load_state_dict(self, state_dict):
        super().load_state_dict(state_dict)
        for k in self._KNN_KEYS:
            setattr(self, k, state_dict[k])

    def hparam_state_dict(self):
        d = super().hparam_state_dict()
        d.update({"k": self.k, "model": "knn"})
        return d
