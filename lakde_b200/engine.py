"""Fused batch VI on a fixed pair pattern.

One VI iteration updates all N kernels at once (the reference's schedule at
block_size = N, lakde/kdes.py:64-67 with one block) and restricts the E-step
to a fixed pattern of candidate pairs (kernel n, point m) held in CSR form
grouped by kernel.  With the all-pairs pattern this is the reference
algorithm itself; with the kNN pattern it is the reference E-step restricted
to those pairs.

An iteration is four launches of the sm_100a library and a few element-wise
updates, with no host synchronisation:

    mstep            S_n, nu_n from r over the pattern          (local_adaptive_kde.py:66-81)
    posterior_factor FP64 jittered Cholesky, W_triu, logdet_W,
                     trace term for the b update                 (local_adaptive_kde.py:83-96)
    estep_logrho     log rho on the pattern                      (local_adaptive_kde.py:36-44)
    estep_normalise  per-point normaliser, threshold, rebalance  (local_adaptive_kde.py:120-181)

and can be captured in a CUDA graph and replayed.  Device-side failures of
the jitter ladder are accumulated into a flag checked by ``check_errors``.
"""

import math

import torch

from . import kernels as K
from .linalg_util import lgamma, mvdigamma, mvlgamma
from .sparse_util import PairPattern

LOG2 = math.log(2.0)


class FusedVI:
    """State and iteration of the locally adaptive models on a pair pattern."""

    def __init__(self, X, pattern, nu_0, a_0, b_0, threshold, init_k, init_graph, precision="auto"):
        self.X = X
        self.N, self.D = X.shape
        self.dtype = X.dtype
        self.device = X.device
        self.pattern = pattern
        self.nu_0 = float(nu_0)
        self.nu_0_t = torch.full((1,), self.nu_0, dtype=self.dtype, device=self.device)
        self.a_0 = a_0
        self.b_0 = b_0
        self.b_0_f = float(b_0)  # host copies: no device read inside a captured step
        self.a_0_f = float(a_0)
        self.threshold = float(threshold or 0.0)
        self.eps = torch.finfo(self.dtype).eps
        N, D = self.N, self.D
        new = lambda *s: torch.empty(*s, dtype=self.dtype, device=self.device)  # noqa: E731
        self.r = self._initial_responsibilities(init_graph, init_k)
        self.c = torch.full((N,), -math.inf, dtype=self.dtype, device=self.device)
        self.rsum = torch.zeros(N, dtype=self.dtype, device=self.device)
        self.logrho = new(pattern.nnz)
        self._S = None  # dense S and W_triu, allocated by the paths that use them
        self._U = None
        self.nu = new(N)
        self.logdet_W = new(N)
        self.trace = new(N)
        self.info = torch.zeros(N, dtype=torch.int32, device=self.device)
        self.failed = torch.zeros((), dtype=torch.int32, device=self.device)
        self.W_inv_jitter = torch.zeros(N, dtype=self.dtype, device=self.device)
        self.a = (a_0 + nu_0 * D / 2).expand(N).contiguous()
        self.b = self.a.clone()
        self.graph = None
        self.tuning = None  # launch choices picked by lakde_b200.tuning.tune_engine
        self.err = torch.zeros(1, dtype=torch.int32, device=self.device)
        # "mixed": the E- and M-step contractions on the tensor cores (tcgen05
        # kind::tf32, hi + lo split of the centred differences and of W_triu,
        # fp32 accumulation); "fp32": the plain FP32 kernels.  Factorisations are
        # FP64 either way.  "auto" takes the tensor cores for 8 < D <= 64; at
        # D <= 8 the one-pass register kernel (fp32) is faster.
        if precision == "auto":
            precision = "mixed" if (8 < D <= 64 and self.dtype == torch.float32) else "fp32"
        if precision not in ("mixed", "fp32"):
            raise ValueError(f"unknown precision {precision!r}")
        if precision == "mixed" and not (D <= 64 and self.dtype == torch.float32):
            raise ValueError("precision='mixed' needs float32 data with D <= 64")
        self.precision = precision
        # tensor-core inputs: rows of X padded to 16 bytes (refreshed from X at
        # the start of every step, so writes into X are seen), the atomic row
        # counter of their work queue, W_triu as W cores
        self.queue = torch.zeros(1, dtype=torch.int32, device=self.device)
        self.Xp = None
        self.Wc = None
        if self.dtype == torch.float32 and D <= 64:
            self._Xp_separate = not (D % 4 == 0 and X.is_contiguous() and X.data_ptr() % 16 == 0)
            self.Xp = K.pad_rows(X) if self._Xp_separate else X
            self.Wc = K.w_cores_like(D, N, self.device)

    # ------------------------------------------------------------------ setup
    def _initial_responsibilities(self, init_graph, init_k):
        """r = 1 / init_k on the pairs (init_graph[m, k], m) (lakde/local_knn_kde.py:113-127)."""
        p = self.pattern
        N = self.N
        r = torch.zeros(p.nnz, dtype=self.dtype, device=self.device)
        keys = p.rows() * N + p.col.long()
        kern = init_graph.reshape(-1).long()
        point = torch.arange(N, device=self.device).repeat_interleave(init_graph.size(1))
        want = kern * N + point
        pos = torch.searchsorted(keys, want)
        ok = (pos < keys.numel()) & (keys[pos.clamp(max=keys.numel() - 1)] == want)
        if not bool(ok.all()):
            raise ValueError("the candidate pattern must contain every initial kNN pair")
        r[pos] = 1.0 / init_k
        return r

    def _tri(self):
        return self.pattern.rowptr, self.pattern.col

    def restore_responsibilities(self, kern, point, values, point_sums=None):
        """r from (kernel, point, value) triples (a checkpoint's COO blocks);
        every pair must lie in the candidate pattern.  rsum = per-point sums of
        r, from the checkpoint when it has them."""
        p = self.pattern
        keys = p.rows() * self.N + p.col.long()
        want = kern.long() * self.N + point.long()
        pos = torch.searchsorted(keys, want)
        ok = (pos < keys.numel()) & (keys[pos.clamp(max=keys.numel() - 1)] == want)
        if not bool(ok.all()):
            raise ValueError(f"{int((~ok).sum())} responsibilities of the checkpoint lie outside the candidate "
                             "pattern; resume with candidates='dense' or a pattern that contains them")
        self.r.zero_()
        self.r[pos] = values.to(self.dtype)
        if point_sums is not None:
            self.rsum.copy_(point_sums.to(self.dtype))
        else:
            self.rsum.zero_().scatter_add_(0, p.col.long(), self.r)

    @property
    def S(self):
        if self._S is None:
            self._S = torch.empty(self.N, self.D, self.D, dtype=self.dtype, device=self.device)
        return self._S

    @property
    def U(self):
        if self._U is None:
            self._U = torch.empty(self.N, self.D, self.D, dtype=self.dtype, device=self.device)
        return self._U

    def refresh_points(self):
        """Copies X into the padded rows the tensor-core kernels read."""
        if self.precision == "mixed" and self._Xp_separate:
            self.Xp.copy_(self.X)

    # whether the trace factor T of _prior() is lower triangular
    _T_lower = False

    def _prior(self):
        """(P, P batch, T) for the posterior factorisation; set by the model."""
        raise NotImplementedError

    # --------------------------------------------------------------- kernels
    # S and P of the mixed path as interleaved 8 x 8 tiles (SP), the trace
    # factor as tiles (Tt): set by models whose prior is per kernel
    SP = None
    Tt = None

    def trace_tiles(self):
        """The trace factor as tiles (tiled path); set by models whose prior is per kernel."""
        return self.Tt

    def mstep(self):
        rowptr, col = self._tri()
        if self.precision == "mixed" and self.SP is not None:
            K.mstep_tc_tiled(rowptr, col, self.r, self.Xp, self.nu_0, self.err, self.SP, self.nu,
                             order=self.pattern.order, queue=self.queue)
        elif self.precision == "mixed":
            K.mstep_tc(rowptr, col, self.r, self.Xp, self.nu_0, self.err, order=self.pattern.order, S=self.S,
                       nu=self.nu, lower_only=True, queue=self.queue)
        else:
            K.mstep(rowptr, col, self.r, self.X, self.nu_0, S=self.S, nu=self.nu)

    def factor(self, with_trace=True):
        mixed = self.precision == "mixed"
        if mixed and self.SP is not None:
            Tt = self.trace_tiles() if with_trace else None
            K.posterior_factor_tiled(self.SP, self.D, self.W_inv_jitter, self.eps, self.nu_0_t, self.a, self.b,
                                     None, self.logdet_W, self.info, T_tiles=Tt,
                                     trace=self.trace if with_trace else None, W_cores=self.Wc)
            torch.minimum(self.failed, self.info.min(), out=self.failed)
            return
        P, T = self._prior()
        K.posterior_factor(
            self.S, self.W_inv_jitter, self.eps, P=P, nu_0=self.nu_0_t, a=self.a, b=self.b,
            T=T if with_trace else None, info=self.info, out=self.U, logdet=self.logdet_W,
            trace=self.trace if with_trace else None, T_lower=self._T_lower, W_cores=self.Wc if mixed else None,
        )
        torch.minimum(self.failed, self.info.min(), out=self.failed)

    def estep_numerators(self):
        """log rho of every pair of the pattern (the E-step before the normaliser)."""
        rowptr, col = self._tri()
        if self.precision == "mixed":
            K.estep_tc(rowptr, col, self.Xp, self.Wc, self.nu, self.logdet_W, self.err, order=self.pattern.order,
                       out=self.logrho, queue=self.queue)
        else:
            K.estep_logrho(rowptr, col, self.X, self.U, self.nu, self.logdet_W, out=self.logrho)

    def estep(self, mode):
        self.estep_numerators()
        K.estep_normalise(self.pattern.cptr, self.pattern.pos, self.logrho, self.r, self.c, self.rsum, mode,
                          self.threshold)

    _STATE = ("r", "c", "rsum", "b", "W_inv_jitter", "nu", "logdet_W")

    def snapshot(self):
        """Copies of the iteration state (to rerun iterations from one point)."""
        keys = self._STATE + tuple(k for k in ("sigma_0_lambda_mm_trace", "W_shared_triu") if hasattr(self, k))
        return {k: getattr(self, k).clone() for k in keys}

    def restore(self, snap):
        for k, v in snap.items():
            getattr(self, k).copy_(v)

    def check_errors(self):
        if int(self.failed) != 0:
            raise RuntimeError("Stabilization did not converge")
        if int(self.err) != 0:
            raise RuntimeError("a tensor-core completion wait timed out; results of this fit are invalid")

    # ------------------------------------------------------------ prediction
    def log_pred_density(self, Y):
        """lakde/local_adaptive_kde.py:200-223: posterior from the current r, then
        the fused Student-t mixture kernel.  S and the factorisation are
        recomputed into buffers the next iteration overwrites first (the S
        halves of SP or S, and the W cores or W_triu), so no per-kernel matrices
        are allocated; nu and logdet_W of the model are left as they are."""
        nu = torch.empty_like(self.nu)
        logdet = torch.empty_like(self.logdet_W)
        info = torch.empty_like(self.info)
        rowptr, col = self._tri()
        if self.precision == "mixed":
            self.refresh_points()
            if self.SP is not None:
                K.mstep_tc_tiled(rowptr, col, self.r, self.Xp, self.nu_0, self.err, self.SP, nu,
                                 order=self.pattern.order, queue=self.queue)
                K.posterior_factor_tiled(self.SP, self.D, self.W_inv_jitter, self.eps, self.nu_0_t, self.a, self.b,
                                         None, logdet, info, W_cores=self.Wc)
            else:
                K.mstep_tc(rowptr, col, self.r, self.Xp, self.nu_0, self.err, order=self.pattern.order, S=self.S,
                           nu=nu, lower_only=True, queue=self.queue)
                P, _ = self._prior()
                K.posterior_factor(self.S, self.W_inv_jitter, self.eps, P=P, nu_0=self.nu_0_t, a=self.a, b=self.b,
                                   info=info, out=self.U, logdet=logdet, W_cores=self.Wc)
            torch.minimum(self.failed, info.min(), out=self.failed)
            lc = K.pred_coeff(nu, logdet, self.D)
            return K.log_pred_density_tc(self.Xp, self.Wc, nu, lc, Y.to(self.dtype), self.err)
        # S and W_triu into the engine's own buffers (the next step rewrites them first)
        K.mstep(rowptr, col, self.r, self.X, self.nu_0, S=self.S, nu=nu)
        P, _ = self._prior()
        K.posterior_factor(self.S, self.W_inv_jitter, self.eps, P=P, nu_0=self.nu_0_t, a=self.a, b=self.b,
                           logdet=logdet, info=info, out=self.U)
        torch.minimum(self.failed, info.min(), out=self.failed)
        lc = K.pred_coeff(nu, logdet, self.D)
        return K.log_pred_density(self.X, self.U, nu, lc, Y.to(self.dtype))

    def posterior_factors(self):
        """(W_triu, nu, logdet_W) as log_pred_density recomputes them."""
        S = torch.empty_like(self.S)
        nu = torch.empty_like(self.nu)
        rowptr, col = self._tri()
        K.mstep(rowptr, col, self.r, self.X, self.nu_0, S=S, nu=nu)
        P, _ = self._prior()
        W, logdet, info, _, _ = K.posterior_factor(S, self.W_inv_jitter, self.eps, P=P, nu_0=self.nu_0_t, a=self.a,
                                                   b=self.b)
        return W, nu, logdet

    # ---------------------------------------------------------- CUDA graphs
    def step(self):
        raise NotImplementedError

    def capture(self):
        """Captures one iteration in a CUDA graph (after one eager warm-up
        iteration has run on the side stream)."""
        g = torch.cuda.CUDAGraph()
        s = torch.cuda.Stream(device=self.device)
        s.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(s):
            with torch.cuda.graph(g, stream=s):
                self.step()
        torch.cuda.current_stream(self.device).wait_stream(s)
        self.graph = g

    def replay(self):
        self.graph.replay()


class FusedKNN(FusedVI):
    """LocalKNearestKDE on a pair pattern (lakde/local_knn_kde.py)."""

    def __init__(self, X, knn_graph, pattern, nu_0, a_0, b_0, threshold, init_k, precision="auto"):
        super().__init__(X, pattern, nu_0, a_0, b_0, threshold, init_k, knn_graph[:, :init_k], precision)
        self.knn_graph = knn_graph
        N, D = self.N, self.D
        self.sigma_0_jitter = torch.zeros(N, dtype=self.dtype, device=self.device)
        self.logdet_sigma_0 = torch.empty(N, dtype=self.dtype, device=self.device)
        self.sigma_0_lambda_mm_trace = torch.empty(N, dtype=self.dtype, device=self.device)

    def init_prior(self):
        """Sigma0 and its jittered factor (lakde/local_knn_kde.py:195-207).  X
        and the kNN graph are fixed, so the prior is computed once and kept."""
        from .utils import batched_knn_cov

        sigma_0 = batched_knn_cov(self.X, self.X, self.knn_graph.long())
        _, logdet_inv, info, L0, _ = K.posterior_factor(sigma_0, self.sigma_0_jitter, self.eps, want_L=True)
        torch.minimum(self.failed, info.min(), out=self.failed)
        self.logdet_sigma_0.copy_(-logdet_inv)
        sigma_0.diagonal(dim1=-2, dim2=-1).add_(self.sigma_0_jitter[:, None])
        self.sigma_0 = sigma_0
        self.sigma_0_tril = L0
        if self.precision == "mixed" and 8 < self.D <= 64:
            # the tensor-core path reads S and P as interleaved tiles (P halves
            # fixed here) and the trace factor as tiles (packed on first use)
            nt = K.tile_count(self.D)
            self.SP = torch.zeros(self.N, nt * 128, dtype=self.dtype, device=self.device)
            K.pack_tiles(sigma_0, self.SP, 128, 64)

    def trace_tiles(self):
        if self.Tt is None:
            nt = K.tile_count(self.D)
            self.Tt = torch.zeros(self.N, nt * 64, dtype=self.dtype, device=self.device)
            K.pack_tiles(self.sigma_0_tril, self.Tt, 64, 0)
        return self.Tt

    _T_lower = True  # the Cholesky factor of Sigma0

    def _prior(self):
        return self.sigma_0, self.sigma_0_tril

    def kernel_launches(self):
        """The library launches of one iteration as callables by kernel name
        (to time them one by one; the step runs them in this order)."""
        p = self.pattern
        if self.D <= 8 and self.precision == "fp32":
            out = {"vi_rows": lambda: K.vi_rows(
                p.rowptr, p.col, self.r, self.X, self.nu_0, self.a, self.b, self.b_0_f, self.W_inv_jitter, self.eps,
                self.nu, self.logdet_W, self.info, self.logrho, P=self.sigma_0, T=self.sigma_0_tril, order=p.order,
                mm=self.sigma_0_lambda_mm_trace)}
        else:
            mixed = self.precision == "mixed"
            out = {("mstep_tc" if mixed else "mstep"): self.mstep, "posterior_factor": self.factor,
                   ("estep_tc" if mixed else "estep_logrho"): self.estep_numerators}
        out["estep_normalise"] = lambda: K.estep_normalise(p.cptr, p.pos, self.logrho, self.r, self.c, self.rsum, 1,
                                                           self.threshold)
        return out

    def init_summaries(self):
        """lakde/local_knn_kde.py:140-193 at block_size = N."""
        self.init_prior()
        self.refresh_points()
        self.mstep()
        self.factor()
        torch.mul(self.nu, self.trace, out=self.sigma_0_lambda_mm_trace)
        self.estep(mode=0)

    def step(self):
        """lakde/local_knn_kde.py:209-254 at block_size = N."""
        if self.D <= 8 and self.precision == "fp32":
            # M-step, factorisation, summaries, b update and log rho in one pass
            p = self.pattern
            K.vi_rows(p.rowptr, p.col, self.r, self.X, self.nu_0, self.a, self.b, self.b_0_f, self.W_inv_jitter,
                      self.eps, self.nu, self.logdet_W, self.info, self.logrho, P=self.sigma_0, T=self.sigma_0_tril,
                      order=p.order, mm=self.sigma_0_lambda_mm_trace)
            torch.minimum(self.failed, self.info.min(), out=self.failed)
            K.estep_normalise(p.cptr, p.pos, self.logrho, self.r, self.c, self.rsum, 1, self.threshold)
            return
        self.refresh_points()
        self.mstep()
        self.factor()
        self.estep(mode=1)
        torch.mul(self.nu, self.trace, out=self.sigma_0_lambda_mm_trace)
        torch.add(self.sigma_0_lambda_mm_trace * (self.nu_0 / 2), self.b_0, out=self.b)

    def compute_elbo(self):
        """lakde/local_knn_kde.py:256-341 (terms :24-47): one FP64 kernel over
        kernels and points with a fixed reduction order; a 0-dim float64
        device tensor."""
        if getattr(self, "_elbo_out", None) is None:
            self._elbo_out = torch.empty((), dtype=torch.float64, device=self.device)
            self._elbo_ws = torch.empty(K.nat.lib().lakde_knn_elbo_workspace(), dtype=torch.uint8,
                                        device=self.device)
        return K.knn_elbo(self.a, self.b, self.nu, self.logdet_W, self.logdet_sigma_0, self.sigma_0_lambda_mm_trace,
                          self.c, self.a_0_f, self.b_0_f, self.nu_0, self.D, out=self._elbo_out,
                          workspace=self._elbo_ws).clone()


class FusedHier(FusedVI):
    """LocalHierarchicalKDE on a pair pattern (lakde/local_hierarchical_kde.py)."""

    def __init__(self, X, knn_graph, pattern, nu_0, a_0, b_0, threshold, init_k, nu_shared_0, precision="auto"):
        super().__init__(X, pattern, nu_0, a_0, b_0, threshold, init_k, knn_graph[:, :init_k], precision)
        self.nu_shared_0 = float(nu_shared_0)
        N, D = self.N, self.D
        self.W_shared_inv_jitter = torch.zeros(1, dtype=torch.float64, device=self.device)
        from .linalg_util import stabilized_cholesky, tril_inverse
        from .utils import cov

        sigma_0 = cov(X, dtype=torch.float64)
        sigma_0_tril, _ = stabilized_cholesky(sigma_0)
        self.lambda_0_triu = tril_inverse(sigma_0_tril).T
        self.lambda_0 = self.lambda_0_triu @ self.lambda_0_triu.T
        self.nu_shared = self.nu_shared_0 + N * self.nu_0
        # fixed buffer (updated in place, so a captured iteration can replay)
        self.W_shared_triu = (self.nu_0 * sigma_0_tril.T / self.nu_shared).contiguous()
        self.expect_lambda_contribs = torch.zeros(1, D, D, dtype=torch.float64, device=self.device)
        self._sigma_bar = torch.empty(D, D, dtype=self.dtype, device=self.device)
        self._refresh_prior()

    def _refresh_prior(self):
        triu = math.sqrt(self.nu_shared) * self.W_shared_triu
        self._sigma_bar.copy_(triu @ triu.T)

    def _prior(self):
        # the trace term is ||E[Sigma_bar]^T W_triu||_F^2: the reference passes the
        # full matrix E[Sigma_bar] where the knn model passes a triangular factor
        # (lakde/local_hierarchical_kde.py:286-288)
        return self._sigma_bar, self._sigma_bar

    def _lambda_contrib(self, weights):
        """sum_n w_n W_triu_n W_triu_n^T in float64 (lakde/local_hierarchical_kde.py:293-297), one
        library kernel over the model-dtype factors (fixed buffers: the step can be captured)."""
        if getattr(self, "_gram_ws", None) is None:
            self._gram_ws = torch.empty(int(K.nat.lib().lakde_weighted_gram_workspace(self.D)), dtype=torch.uint8,
                                        device=self.device)
            self._gram_out = torch.empty(self.D, self.D, dtype=torch.float64, device=self.device)
        return K.weighted_gram(self.U, weights, out=self._gram_out, workspace=self._gram_ws)

    def kernel_launches(self):
        """The library launches of one iteration as callables by kernel name
        (to time them one by one; the step runs them in this order)."""
        p = self.pattern
        mixed = self.precision == "mixed"
        return {
            ("mstep_tc" if mixed else "mstep"): self.mstep,
            "posterior_factor": self.factor,
            ("estep_tc" if mixed else "estep_logrho"): self.estep_numerators,
            "estep_normalise": lambda: K.estep_normalise(p.cptr, p.pos, self.logrho, self.r, self.c, self.rsum, 1,
                                                         self.threshold),
            "weighted_gram": lambda: self._lambda_contrib(self.nu * (self.a / self.b)),
        }

    def init_summaries(self):
        """lakde/local_hierarchical_kde.py:198-258 at block_size = N."""
        self.refresh_points()
        self.mstep()
        self.factor(with_trace=False)
        e_tau = self.a / self.b
        self.expect_lambda_contribs[0] = self._lambda_contrib(self.nu * e_tau)
        self.estep(mode=0)

    def step(self):
        """lakde/local_hierarchical_kde.py:273-332 at block_size = N."""
        self.refresh_points()
        self.mstep()
        self.factor()
        self.estep(mode=1)
        mm = self.nu * self.trace
        torch.add(mm * (self.nu_0 / 2), self.b_0, out=self.b)
        self.expect_lambda_contribs[0] = self._lambda_contrib(self.nu * (self.a / self.b))
        prec = (self.expect_lambda_contribs.sum(0) * self.nu_0 + self.nu_shared_0 * self.lambda_0).unsqueeze(0)
        W_sh, _, info, _, _ = K.posterior_factor(prec.contiguous(), self.W_shared_inv_jitter,
                                                 torch.finfo(torch.float64).eps)
        torch.minimum(self.failed, info.min(), out=self.failed)
        self.W_shared_triu.copy_(W_sh[0])
        # E[Sigma_bar] follows the shared factor at once, so the next step and
        # log_pred_density both see the current prior
        self._refresh_prior()

    def compute_elbo(self):
        """lakde/local_hierarchical_kde.py:334-461 (terms :25-79), reduced in float64."""
        N, D = self.N, self.D
        dev = self.device
        f = lambda t: t.double()  # noqa: E731
        a, b, nu = f(self.a), f(self.b), f(self.nu)
        a_0 = torch.tensor(float(self.a_0), dtype=torch.float64, device=dev)
        b_0 = torch.tensor(float(self.b_0), dtype=torch.float64, device=dev)
        nu_0 = torch.tensor(self.nu_0, dtype=torch.float64, device=dev)
        nsh0 = torch.tensor(self.nu_shared_0, dtype=torch.float64, device=dev)
        nsh = torch.tensor(self.nu_shared, dtype=torch.float64, device=dev)
        e_tau = a / b
        triu = math.sqrt(self.nu_shared) * self.W_shared_triu
        sigma_bar = triu @ triu.T
        e_log_tau = torch.digamma(a) - torch.log(b)
        e_logdet = mvdigamma(nu / 2, D) + D * LOG2 + f(self.logdet_W)
        lam_sum = self.expect_lambda_contribs.sum(0)
        logdet_sigma_0 = -2 * self.lambda_0_triu.diagonal().log().sum()
        logdet_W_shared = 2 * self.W_shared_triu.diagonal().log().sum()
        e_logdet_sh = mvdigamma(nsh / 2, D) + D * LOG2 + logdet_W_shared
        tr_lam = torch.trace(sigma_bar @ lam_sum)
        tr_lam0 = torch.trace(sigma_bar @ self.lambda_0)
        p_tau = torch.sum(-lgamma(a_0) + a_0 * torch.log(b_0) + (a_0 - 1) * e_log_tau - b_0 * e_tau)
        q_tau = torch.sum(-lgamma(a) + a * torch.log(b) + (a - 1) * e_log_tau - b * e_tau)
        B_p = -nu_0 / 2 * (D * LOG2 - D * e_log_tau - D * torch.log(nu_0) - e_logdet_sh) - mvlgamma(nu_0 / 2, D)
        p_lam = torch.sum(B_p + (nu_0 - D - 1) * e_logdet / 2) - nu_0 * tr_lam / 2
        B_q = -nu / 2 * (f(self.logdet_W) + D * LOG2) - mvlgamma(nu / 2, D)
        q_lam = torch.sum(B_q + (nu - D - 1) * e_logdet / 2 - nu * D / 2)
        p_sh = (-nsh0 / 2 * (logdet_sigma_0 + D * LOG2 - D * torch.log(nsh0)) - mvlgamma(nsh0 / 2, D)
                + (nsh0 - D - 1) * e_logdet_sh / 2 - nsh0 * tr_lam0 / 2)
        q_sh = (-nsh / 2 * (logdet_W_shared + D * LOG2) - mvlgamma(nsh / 2, D) + (nsh - D - 1) * e_logdet_sh / 2
                - nsh * D / 2)
        ll = torch.sum(-D / 2 * math.log(2 * math.pi) + f(self.c))
        return ll + (p_lam - q_lam) - N * math.log(N - 1) + (p_tau - q_tau) + (p_sh - q_sh)


def build_pattern(kind, knn_graph, N, device, counts=None):
    """Candidate pattern: 'knn' (the kNN graph transposed), 'dense' (all pairs),
    'lists' (the first counts[m] neighbours of each point) or a PairPattern."""
    if isinstance(kind, PairPattern):
        return kind
    if kind == "knn":
        return PairPattern.from_knn_graph(knn_graph)
    if kind == "dense":
        return PairPattern.dense(N, device)
    if kind == "lists":
        return PairPattern.from_neighbour_lists(knn_graph, counts)
    raise ValueError(f"unknown candidate pattern {kind!r}")
