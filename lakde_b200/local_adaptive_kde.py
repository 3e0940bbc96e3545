"""Locally adaptive KDE base class (lakde/local_adaptive_kde.py).

Two schedules share the model API:

* ``fused=False`` (default): the reference algorithm exactly -- block
  coordinate ascent over kernel blocks of ``block_size`` with the dense E-step,
  the running normaliser and the rebalance step -- with every numeric kernel
  (scatter covariance, FP64 factorisation, quad forms, predictive density)
  running in the sm_100a library.
* ``fused=True``: batch VI (one block of all N kernels) on a fixed candidate
  pair pattern (``candidates``: "knn", "dense", "lists" or a PairPattern),
  four library launches per iteration, optionally replayed as a CUDA graph
  (see ``lakde_b200.engine``).  With ``candidates="dense"`` it reproduces the
  reference run with block_size = N.
"""

import math
from abc import ABC, abstractmethod

import torch

from . import kernels as K
from .kdes import VIModel
from .linalg_util import chol_logdet, lgamma, logsubexp, mvdigamma, xlogx
from .sparse_util import cat_sparse


def expect_log_p_tau(a_0, b_0, expect_tau, expect_log_tau):
    """lakde/local_adaptive_kde.py:21-26."""
    return torch.sum(-lgamma(a_0) + a_0 * torch.log(b_0) + (a_0 - 1) * expect_log_tau - b_0 * expect_tau)


def expect_log_q_tau(a, b, expect_tau, expect_log_tau):
    """lakde/local_adaptive_kde.py:29-33."""
    return torch.sum(-lgamma(a) + a * torch.log(b) + (a - 1) * expect_log_tau - b * expect_tau)


def calc_log_rho_block(X_test, X_train, nu, W_triu, logdet_W):
    """log rho[n, m] = 0.5 E[log|Lambda_n|] - nu_n / 2 Q[n, m] (lakde/local_adaptive_kde.py:36-44)."""
    D = X_test.size(-1)
    expect_logdet_lambda = mvdigamma(nu / 2, D) + D * math.log(2) + logdet_W
    Q = K.chol_quad_form(W_triu, X_train, X_test)
    Q *= (-0.5 * nu)[:, None]
    Q += (0.5 * expect_logdet_lambda)[:, None]
    return Q


class LocallyAdaptiveKDE(VIModel, ABC):
    def __init__(self, nu_0, a_0, b_0, block_size, verbose, logs, fused=False, candidates="knn", cuda_graph=True):
        super().__init__(block_size, verbose, logs)
        self.nu_0 = nu_0
        self.nu = None
        self.a_0 = a_0
        self.b_0 = b_0
        self.a = None
        self.b = None
        self.rnm_blocks = None
        self.rnm_log_consts = None
        self.logdet_W = None
        self.rnm_active_contribs = None
        self.W_inv_jitter = None
        self.fused = fused
        self.candidates = candidates
        self.cuda_graph = cuda_graph
        self.engine = None

    # ------------------------------------------------------------------ blocks
    def num_blocks(self, N):
        return 1 if self.fused else (N - 1) // self.block_size + 1

    def _span(self, block_idx):
        s = block_idx * self.block_size
        return s, s + self.block_size

    def calc_posterior_contribs(self, X, block_idx):
        """S and nu of one kernel block from its COO (lakde/local_adaptive_kde.py:66-81)."""
        s, e = self._span(block_idx)
        X_train = X[s:e]
        (row, col), values = self.rnm_blocks[block_idx]
        rowptr = K.ind2ptr(row.long().contiguous(), X_train.size(0), out=torch.empty(
            X_train.size(0) + 1, dtype=torch.int64, device=X.device))
        return K.mstep(rowptr, col.contiguous(), values.contiguous(), X, float(self.nu_0), kernel_offset=s)

    def calc_posterior(self, block_idx, sigma_0, W_inv_contrib):
        """W_triu = chol(nu_0 E[tau] Sigma0 + S)^-T with the jitter ladder (lakde/local_adaptive_kde.py:83-96)."""
        s, e = self._span(block_idx)
        jitter = self.W_inv_jitter[s:e]
        W_triu, _, info, _, _ = K.posterior_factor(
            W_inv_contrib, jitter, torch.finfo(W_inv_contrib.dtype).eps, P=sigma_0, nu_0=self.nu_0, a=self.a[s:e],
            b=self.b[s:e],
        )
        if bool((info != 0).any()):
            raise RuntimeError("Stabilization did not converge")
        return W_triu

    def partial_expectation_step(self, X, block_idx, W_triu, nu, update_normalization=True, sparsity_threshold=None):
        """Dense E-step of one kernel block against all points (lakde/local_adaptive_kde.py:98-154)."""
        N, D = X.shape
        s, e = self._span(block_idx)
        X_train = X[s:e]
        logdet_W = chol_logdet(W_triu)
        rnm_log_consts = self.rnm_log_consts
        old_log_consts = rnm_log_consts
        blocks = []
        if update_normalization:
            rnm_log_consts = rnm_log_consts.clone()
            (_, col), values = self.rnm_blocks[block_idx]
            old_sums = X.new_zeros(N).scatter_add_(0, col.long(), values)
            old_contribs = torch.log(old_sums) + old_log_consts
        for bj, j in enumerate(range(0, N, self.block_size)):
            X_test = X[j : j + self.block_size]
            log_rho = calc_log_rho_block(X_test, X_train, nu, W_triu, logdet_W)
            if block_idx == bj:
                log_rho.diagonal().fill_(-math.inf)
            if update_normalization:
                sl = slice(j, j + self.block_size)
                torch.logaddexp(
                    logsubexp(old_log_consts[sl], old_contribs[sl]),
                    torch.logsumexp(log_rho, dim=0),
                    out=rnm_log_consts[sl],
                )
            r = torch.exp_(log_rho.sub_(rnm_log_consts[j : j + self.block_size]))
            if sparsity_threshold:
                r = torch.threshold_(r, sparsity_threshold, 0)
            idx = torch.nonzero(r).T.contiguous()
            blocks.append((idx.to(torch.int32), r[idx.unbind()]))
        indices, values = cat_sparse(*zip(*blocks), self.block_size, dim=1)
        perm = torch.argsort(indices[0].long() * N + indices[1].long())
        indices, values = indices[:, perm], values[perm]
        if update_normalization:
            return indices, values, rnm_log_consts
        return indices, values

    def rebalance_responsibilities_(self, X, block_idx, rnm_log_consts):
        """Rescale the other blocks and renormalise so sum_n r_nm = 1 (lakde/local_adaptive_kde.py:156-181)."""
        N = X.size(0)
        finfo = torch.finfo(X.dtype)
        coeff = torch.clamp_(torch.exp(self.rnm_log_consts - rnm_log_consts), min=finfo.tiny, max=finfo.max)
        sums = X.new_zeros(N)
        for bi in range(len(self.rnm_blocks)):
            (_, col), values = self.rnm_blocks[bi]
            col = col.long()
            if bi != block_idx:
                values *= coeff[col]
            sums.scatter_add_(0, col, values)
        sums = torch.clamp_min(sums, finfo.eps)
        rnm_log_consts += sums.log()
        coeff = torch.clamp_(torch.reciprocal(sums), min=finfo.tiny, max=finfo.max)
        for bi in range(len(self.rnm_blocks)):
            (_, col), values = self.rnm_blocks[bi]
            values *= coeff[col.long()]
        return rnm_log_consts

    # ------------------------------------------------------------- fused path
    def _sync_from_engine(self):
        """Expose the engine state under the reference attribute names."""
        eng = self.engine
        self.nu = eng.nu
        self.a = eng.a
        self.b = eng.b
        self.rnm_log_consts = eng.c
        self.logdet_W = eng.logdet_W
        self.W_inv_jitter = eng.W_inv_jitter

    def _fused_step(self):
        eng = self.engine
        if (getattr(self, "autotune", False) and self._eager_steps >= 1 and getattr(eng, "tuning", None) is None
                and hasattr(eng, "kernel_launches")):
            # after one eager iteration (every buffer allocated), before the capture
            from .tuning import tune_engine

            eng.tuning = tune_engine(eng)
        if self.cuda_graph and eng.graph is None and self._eager_steps >= 1:
            eng.capture()
        if eng.graph is not None:
            eng.replay()
        else:
            eng.step()
            self._eager_steps += 1
        self._sync_from_engine()

    def check_errors_(self):
        if self.engine is not None:
            self.engine.check_errors()

    @property
    def responsibilities(self):
        """(PairPattern, r) of the fused path."""
        return self.engine.pattern, self.engine.r

    def fused_rnm_blocks(self):
        """Responsibilities of the fused path in the reference COO layout (one block)."""
        return self.engine.pattern.to_blocks(self.engine.r, self.engine.N)

    # ---------------------------------------------------------------- outputs
    def data_log_likelihood_no_rnm(self, X):
        N, D = X.shape
        return -D / 2 * math.log(2 * math.pi) + self.rnm_log_consts

    def data_log_likelihood(self, X):
        ll = self.data_log_likelihood_no_rnm(X).clone()
        if self.fused:
            p, r = self.responsibilities
            ll.scatter_add_(0, p.col.long(), xlogx(r))
            return ll
        for bi in range(len(self.rnm_blocks)):
            (_, col), values = self.rnm_blocks[bi]
            ll.scatter_add_(0, col.long(), xlogx(values))
        return ll

    @abstractmethod
    def calc_prior_cov(self, X, bi):
        pass

    def log_pred_density(self, X, Y):
        """Predictive log density of Y (lakde/local_adaptive_kde.py:200-223)."""
        if self.fused:
            out = self.engine.log_pred_density(Y)
            self._sync_from_engine()
            return out
        N_train, D = X.shape
        acc = Y.new_full((Y.size(0),), -math.inf)
        for bi in range(self.num_blocks(N_train)):
            s, e = self._span(bi)
            W_inv_contrib, nu = self.calc_posterior_contribs(X, bi)
            sigma_0, _ = self.calc_prior_cov(X, bi)
            W_triu = self.calc_posterior(bi, sigma_0, W_inv_contrib)
            lc = K.pred_coeff(nu, chol_logdet(W_triu).contiguous(), D)
            # the kernel returns -log(block size) + logsumexp over the block
            part = K.log_pred_density(X[s:e].contiguous(), W_triu, nu, lc, Y)
            part = part + math.log(W_triu.size(0))
            torch.logaddexp(acc, part, out=acc)
        return -math.log(N_train) + acc

    def sample(self, X, n):
        """Draws n points from the predictive Student-t mixture (lakde/local_adaptive_kde.py:225-270)."""
        N, D = X.shape
        idx = torch.randint(N, (n,), device=X.device)
        out = X.new_empty(n, D)
        if self.fused:
            W, nu, _ = self.engine.posterior_factors()
        else:
            Ws, nus = [], []
            for bi in range(self.num_blocks(N)):
                S, nu_b = self.calc_posterior_contribs(X, bi)
                sigma_0, _ = self.calc_prior_cov(X, bi)
                Ws.append(self.calc_posterior(bi, sigma_0, S))
                nus.append(nu_b)
            W, nu = torch.cat(Ws), torch.cat(nus)
        dof = nu[idx] + 1 - D
        # x = x_n + y / sqrt(u / dof), y ~ N(0, (dof W)^-1), u ~ Chi2(dof)
        z = torch.randn(n, D, dtype=X.dtype, device=X.device)
        y = torch.linalg.solve_triangular(W[idx].mT * dof.sqrt()[:, None, None], z.unsqueeze(-1), upper=False)
        y = y.squeeze(-1)
        u = torch.clamp_min(torch.distributions.Chi2(df=dof).sample(), torch.finfo(X.dtype).eps)
        out[:] = X[idx] + y / torch.sqrt(u / dof)[:, None]
        return out

    # ------------------------------------------------------------------- state
    _STATE_KEYS = ("nu_0", "nu", "a_0", "b_0", "a", "b", "rnm_blocks", "rnm_log_consts", "logdet_W",
                   "rnm_active_contribs", "W_inv_jitter")

    def state_dict(self):
        """The reference's keys (lakde/local_adaptive_kde.py:287-305); the fused
        path writes its responsibilities as one COO block and adds the per-point
        sums of r (``rnm_point_sums``), so a resumed fit continues bit for bit."""
        d = super().state_dict()
        if self.fused and self.engine is not None:
            self.rnm_blocks = self.fused_rnm_blocks()
            self.rnm_active_contribs = torch.count_nonzero(self.engine.r)
            d["rnm_point_sums"] = self.engine.rsum.clone()
        d.update({k: getattr(self, k) for k in self._STATE_KEYS})
        return d

    def load_state_dict(self, state_dict):
        """Restores the reference's keys (lakde/local_adaptive_kde.py:272-285).
        The next ``fit`` continues from this state (``resume_``): the block
        schedule uses the COO blocks as they are; the fused schedule rebuilds
        its engine and scatters the COO blocks (any block size, the reference's
        included) into its candidate pattern."""
        super().load_state_dict(state_dict)
        for k in self._STATE_KEYS:
            setattr(self, k, state_dict[k])
        self.engine = None
        self._point_sums = state_dict.get("rnm_point_sums")

    def _resume_tensors(self, X, keys):
        dev = X.device
        for k in keys:
            v = getattr(self, k, None)
            if torch.is_tensor(v):
                setattr(self, k, v.to(dev))
        if self.rnm_blocks is not None:  # None while a fused engine holds the responsibilities
            self.rnm_blocks = [(ind.to(dev), val.to(device=dev, dtype=X.dtype)) for ind, val in self.rnm_blocks]

    def _restore_engine_state(self, eng):
        """Responsibilities and per-kernel / per-point state of a checkpoint into a
        freshly built engine (whose prior is already computed)."""
        kern, point, vals = [], [], []
        for bi, (ind, val) in enumerate(self.rnm_blocks):
            kern.append(ind[0].long() + bi * self.block_size)
            point.append(ind[1].long())
            vals.append(val)
        eng.restore_responsibilities(torch.cat(kern), torch.cat(point), torch.cat(vals), self._point_sums)
        for name, src in (("c", self.rnm_log_consts), ("a", self.a), ("b", self.b), ("nu", self.nu),
                          ("logdet_W", self.logdet_W), ("W_inv_jitter", self.W_inv_jitter)):
            getattr(eng, name).copy_(src.to(eng.dtype))

    def hparam_state_dict(self):
        d = super().hparam_state_dict()
        d.update({"nu_0": float(self.nu_0)})
        return d
