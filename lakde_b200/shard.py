"""Kernels sharded over devices: LocalKNearestKDE's batch VI on several GPUs.

One process per GPU.  The N kernels (rows of the kernel-major pair pattern)
are split into contiguous ranges of about equal pair counts; every rank keeps
X (all points) and the per-point state (normaliser c, row sums rsum), and the
per-kernel state of its own range only.  Per iteration each rank runs the
M-step, the FP64 factorisation and the E-step numerators of its kernels with
no communication; the one exchange is the per-point normaliser, whose
logsumexp and row sums run over the kernels of every rank:

    stage 0  local max of log rho per point      -> all-reduce max
    stage 1  local sum of exp(log rho - max)     -> all-reduce sum
    stage 2  c_new, local sum of the new r       -> all-reduce sum
    stage 3  c, r rescaled, local row sums       -> all-reduce sum

(N floats each; lakde/local_adaptive_kde.py:120-181 is the single-device
pass these stages split).  The ELBO adds per-kernel sums over ranks;
log_pred_density combines the per-rank logsumexp over kernels with a max and
a sum all-reduce.  The kernel ranges are fixed, so no kernel state moves.

The per-shard arithmetic is reached through an ``ops`` object (the library's
CUDA kernels by default, ``CudaShardOps``) and the collectives through a
``comm`` object (``TorchComm`` over torch.distributed: NCCL between GPUs).
"""

import math

import torch

from .sparse_util import PairPattern



def balanced_ranges(rowptr, world):
    """Contiguous kernel ranges [(lo, hi)] with about equal pair counts."""
    rp = rowptr.detach().to("cpu", torch.int64)
    N = rp.numel() - 1
    total = int(rp[-1])
    targets = torch.tensor([(total * g + world // 2) // world for g in range(world + 1)], dtype=torch.int64)
    cut = torch.searchsorted(rp, targets).clamp(0, N).tolist()
    cut[0], cut[-1] = 0, N
    for g in range(1, world + 1):
        cut[g] = max(cut[g], cut[g - 1])
    return [(cut[g], cut[g + 1]) for g in range(world)]


def shard_pattern(pattern, lo, hi):
    """The pairs of kernels lo..hi-1 as a pattern of hi - lo kernel rows over
    all points (point-major view over these pairs only).  The rows keep the
    global CSR order (ascending point within a kernel)."""
    p0, p1 = int(pattern.rowptr[lo]), int(pattern.rowptr[hi])
    n, N = hi - lo, pattern.n_points
    rowptr = (pattern.rowptr[lo : hi + 1] - p0).contiguous()
    col = pattern.col[p0:p1].contiguous()
    kern = torch.repeat_interleave(torch.arange(n, device=pattern.device), rowptr[1:] - rowptr[:-1])
    point = col.long()
    pos = torch.argsort(point * max(n, 1) + kern)
    cptr = torch.zeros(N + 1, dtype=torch.int64, device=pattern.device)
    cptr[1:] = torch.cumsum(torch.bincount(point, minlength=N), 0)
    pos = pos.to(torch.int32) if point.numel() < 2**31 else pos
    rank = None if pattern.rank is None else pattern.rank[p0:p1]
    return PairPattern(rowptr, col, cptr, pos, n, N, rank)


class TorchComm:
    """All-reduces over a torch.distributed process group."""

    def __init__(self, group=None):
        import torch.distributed as dist

        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)

    def max_(self, t):
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX, group=self.group)

    def sum_(self, t):
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM, group=self.group)


class LocalComm:
    """A world of one (no communication)."""

    rank, world = 0, 1

    def max_(self, t):
        pass

    def sum_(self, t):
        pass


class CudaShardOps:
    """The per-shard arithmetic on this library's kernels."""

    def __init__(self):
        from . import kernels

        self.K = kernels
        self._Xp = None

    def _rows(self, X):
        """X with 16-byte aligned rows for the tensor-core kernels: X itself, or a
        padded copy refreshed from X on every call."""
        D = X.size(1)
        if D % 4 == 0 and X.is_contiguous() and X.data_ptr() % 16 == 0:
            return X
        if self._Xp is None or self._Xp.shape != X.shape or self._Xp.device != X.device:
            self._Xp = self.K.pad_rows(X)
        else:
            self._Xp.copy_(X)
        return self._Xp

    def prior(self, X, graph_rows, lo, jitter, eps):
        """Sigma0 of kernels lo.. (with jitter), its factor, log det and the
        worst factorisation status (lakde/local_knn_kde.py:195-207)."""
        from .utils import batched_knn_cov

        n = graph_rows.size(0)
        sigma_0 = batched_knn_cov(X, X[lo : lo + n], graph_rows.long())
        _, logdet_inv, info, L0, _ = self.K.posterior_factor(sigma_0, jitter, eps, want_L=True)
        sigma_0.diagonal(dim1=-2, dim2=-1).add_(jitter[:, None])
        return sigma_0, L0, -logdet_inv, info.min()

    def mstep(self, pat, r, X, lo, nu_0, S, nu, precision, err, queue=None):
        if precision == "mixed":
            self.K.mstep_tc(pat.rowptr, pat.col, r, self._rows(X), nu_0, err, order=pat.order, S=S, nu=nu,
                            lower_only=True, kernel_offset=lo, queue=queue)
        else:
            self.K.mstep(pat.rowptr, pat.col, r, X, nu_0, kernel_offset=lo, S=S, nu=nu)

    def factor(self, S, jitter, eps, P, nu_0, a, b, T, U, logdet, trace, info, W_cores=None):
        self.K.posterior_factor(S, jitter, eps, P=P, nu_0=nu_0, a=a, b=b, T=T, info=info, out=U, logdet=logdet,
                                trace=trace, T_lower=True, W_cores=W_cores)

    def estep(self, pat, X, lo, U, nu, logdet, out, precision, err, W_cores=None, queue=None):
        if precision == "mixed":
            Wc = W_cores if W_cores is not None else self.K.pack_w_cores(U)
            self.K.estep_tc(pat.rowptr, pat.col, self._rows(X), Wc, nu, logdet, err, order=pat.order, out=out,
                            kernel_offset=lo, queue=queue)
        else:
            self.K.estep_logrho(pat.rowptr, pat.col, X, U, nu, logdet, kernel_offset=lo, out=out)

    def normalise_stage(self, stage, pat, logrho, r, c, rsum, red, red2, mode, threshold):
        self.K.estep_normalise_stage(stage, pat.cptr, pat.pos, logrho, r, c, rsum, red, red2, mode, threshold)

    def elbo_kernel_terms(self, a, b, nu, logdet_W, logdet_sigma_0, mm, D, a_0, b_0, nu_0):
        """float64 sum of the ELBO's per-kernel terms of this shard's kernels, shape (1,)."""
        if a.numel() == 0:
            return torch.zeros(1, dtype=torch.float64, device=a.device)
        return self.K.knn_elbo_parts(D, a_0, b_0, nu_0, a=a, b=b, nu=nu, logdet_W=logdet_W,
                                     logdet_sigma_0=logdet_sigma_0, mm=mm).reshape(1)

    def elbo_point_terms(self, c, D, tail, a_0, b_0, nu_0):
        """float64 sum of the ELBO's per-point terms plus tail (0-dim)."""
        return self.K.knn_elbo_parts(D, a_0, b_0, nu_0, c=c, tail=tail)

    def vi_rows(self, pat, r, X, lo, nu_0, a, b, b_0, jitter, eps, nu, logdet, info, logrho, P, T, mm):
        """M-step, factorisation, b update and log rho of this shard's rows in
        one pass (D <= 8)."""
        self.K.vi_rows(pat.rowptr, pat.col, r, X, nu_0, a, b, b_0, jitter, eps, nu, logdet, info, logrho, P=P, T=T,
                       order=pat.order, mm=mm, kernel_offset=lo)

    def pred(self, Xk, U, nu, logdet, Y, precision, err):
        """-log n + logsumexp over these n kernels, per query."""
        lc = self.K.pred_coeff(nu, logdet, Xk.size(1))
        if precision == "mixed":
            return self.K.log_pred_density_tc(Xk, self.K.pack_w_cores(U), nu, lc, Y, err)
        return self.K.log_pred_density(Xk, U, nu, lc, Y)


class ShardedKNN:
    """LocalKNearestKDE's fused batch VI with kernels sharded over ranks.

    ``pattern`` is the global pair pattern (every rank builds the same one);
    the rank keeps the rows of its kernel range.  Per-point state (c, rsum)
    is identical on every rank after each iteration.
    """

    def __init__(self, X, knn_graph, pattern, nu_0, a_0, b_0, threshold, init_k, comm=None, ops=None,
                 precision="auto"):
        self.comm = comm if comm is not None else LocalComm()
        self.ops = ops if ops is not None else CudaShardOps()
        self.X = X
        self.N, self.D = X.shape
        N, D = self.N, self.D
        self.dtype, self.device = X.dtype, X.device
        self.ranges = balanced_ranges(pattern.rowptr, self.comm.world)
        self.lo, self.hi = self.ranges[self.comm.rank]
        self.n = self.hi - self.lo
        self.pat = shard_pattern(pattern, self.lo, self.hi)
        self.knn_rows = knn_graph[self.lo : self.hi]
        self.nu_0 = float(nu_0)
        self.nu_0_t = torch.full((1,), self.nu_0, dtype=self.dtype, device=self.device)
        self.a_0, self.b_0 = float(a_0), float(b_0)
        self.threshold = float(threshold or 0.0)
        self.eps = torch.finfo(self.dtype).eps
        if precision == "auto":
            precision = "mixed" if (8 < D <= 64 and self.dtype == torch.float32 and X.is_cuda) else "fp32"
        self.precision = precision
        n = self.n
        new = lambda *s: torch.empty(*s, dtype=self.dtype, device=self.device)  # noqa: E731
        self.r = self._initial_responsibilities(knn_graph, init_k)
        self.c = torch.full((N,), -math.inf, dtype=self.dtype, device=self.device)
        self.rsum = torch.zeros(N, dtype=self.dtype, device=self.device)
        self.red, self.red2 = new(N), new(N)
        self.logrho = new(self.pat.nnz)
        self.S, self.U = new(n, D, D), new(n, D, D)
        self.nu, self.logdet_W, self.trace = new(n), new(n), new(n)
        self.info = torch.zeros(n, dtype=torch.int32, device=self.device)
        self.W_inv_jitter = torch.zeros(n, dtype=self.dtype, device=self.device)
        self.sigma_0_jitter = torch.zeros(n, dtype=self.dtype, device=self.device)
        self.a = torch.full((n,), self.a_0 + self.nu_0 * D / 2, dtype=self.dtype, device=self.device)
        self.b = self.a.clone()
        self.mm = new(n)
        self.err = torch.zeros(1, dtype=torch.int32, device=self.device)
        # tensor-core path: W_triu of the shard's kernels as W cores, the work-queue counter
        self.Wc = self.queue = None
        if precision == "mixed":
            from . import kernels

            self.Wc = kernels.w_cores_like(D, max(n, 1), self.device)[:n]
            self.queue = torch.zeros(1, dtype=torch.int32, device=self.device)
        self.failed = torch.zeros((), dtype=torch.int32, device=self.device)

    def _initial_responsibilities(self, knn_graph, init_k):
        """r = 1 / init_k on the pairs (n, m) with n among the first init_k
        neighbours of m (lakde/local_knn_kde.py:113-127)."""
        p = self.pat
        if p.rank is not None:
            return torch.where(p.rank < init_k, 1.0 / init_k, 0.0).to(self.dtype)
        r = torch.zeros(p.nnz, dtype=self.dtype, device=self.device)
        keys = p.rows() * self.N + p.col.long()
        kern = knn_graph[:, :init_k].reshape(-1).long()
        point = torch.arange(self.N, device=self.device).repeat_interleave(init_k)
        mine = (kern >= self.lo) & (kern < self.hi)
        want = (kern[mine] - self.lo) * self.N + point[mine]
        pos = torch.searchsorted(keys, want)
        ok = (pos < keys.numel()) & (keys[pos.clamp(max=max(keys.numel() - 1, 0))] == want)
        if not bool(ok.all()):
            raise ValueError("the candidate pattern must contain every initial kNN pair")
        r[pos] = 1.0 / init_k
        return r

    # ------------------------------------------------------------- iteration
    def _mstep(self):
        self.ops.mstep(self.pat, self.r, self.X, self.lo, self.nu_0, self.S, self.nu, self.precision, self.err,
                       **self._tc_kw())

    def _factor(self):
        self.ops.factor(self.S, self.W_inv_jitter, self.eps, self.sigma_0, self.nu_0_t, self.a, self.b,
                        self.sigma_0_tril, self.U, self.logdet_W, self.trace, self.info,
                        **({"W_cores": self.Wc} if self.Wc is not None else {}))
        if self.n:
            torch.minimum(self.failed, self.info.min(), out=self.failed)

    def _estep(self, mode):
        self.ops.estep(self.pat, self.X, self.lo, self.U, self.nu, self.logdet_W, self.logrho, self.precision,
                       self.err, **self._tc_kw(W_cores=self.Wc))
        self._normalise(mode)

    def _tc_kw(self, **kw):
        """Extra arguments of the tensor-core path (none for the plain kernels)."""
        if self.precision != "mixed":
            return {}
        kw["queue"] = self.queue
        return kw

    def _normalise(self, mode):
        """The per-point pass, reduced over the ranks between its stages."""
        args = (self.pat, self.logrho, self.r, self.c, self.rsum, self.red, self.red2, mode, self.threshold)
        self.ops.normalise_stage(0, *args)
        self.comm.max_(self.red)
        self.ops.normalise_stage(1, *args)
        self.comm.sum_(self.red2)
        self.ops.normalise_stage(2, *args)
        self.comm.sum_(self.red2)
        self.ops.normalise_stage(3, *args)
        self.comm.sum_(self.rsum)

    def init_summaries(self):
        """lakde/local_knn_kde.py:140-193 at block_size = N."""
        if self.n:
            self.sigma_0, self.sigma_0_tril, self.logdet_sigma_0, worst = self.ops.prior(
                self.X, self.knn_rows, self.lo, self.sigma_0_jitter, self.eps)
            torch.minimum(self.failed, worst, out=self.failed)
        else:
            self.sigma_0, self.sigma_0_tril = torch.empty_like(self.S), torch.empty_like(self.S)
            self.logdet_sigma_0 = torch.empty_like(self.nu)
        self._mstep()
        self._factor()
        torch.mul(self.nu, self.trace, out=self.mm)
        self._estep(mode=0)

    def step(self):
        """lakde/local_knn_kde.py:209-254 at block_size = N."""
        if self.D <= 8 and hasattr(self.ops, "vi_rows"):
            # the shard's rows in one fused pass, then the reduced per-point pass
            if self.n:
                self.ops.vi_rows(self.pat, self.r, self.X, self.lo, self.nu_0, self.a, self.b, self.b_0,
                                 self.W_inv_jitter, self.eps, self.nu, self.logdet_W, self.info, self.logrho,
                                 self.sigma_0, self.sigma_0_tril, self.mm)
                torch.minimum(self.failed, self.info.min(), out=self.failed)
            self._normalise(1)
            return
        self._mstep()
        self._factor()
        self._estep(mode=1)
        torch.mul(self.nu, self.trace, out=self.mm)
        torch.add(self.mm * (self.nu_0 / 2), self.b_0, out=self.b)

    def check_errors(self):
        """Raises if a factorisation or a tensor-core wait failed on any rank."""
        flags = torch.stack([(self.failed < 0).to(torch.float64), (self.err != 0).any().to(torch.float64)])
        self.comm.sum_(flags)
        if float(flags[0]) > 0:
            raise RuntimeError("Stabilization did not converge")
        if float(flags[1]) > 0:
            raise RuntimeError("a tensor-core completion wait timed out")

    # ------------------------------------------------------------- read-outs
    def compute_elbo(self):
        """lakde/local_knn_kde.py:256-341 in float64: per-kernel terms summed
        over the ranks, per-point terms (identical on every rank) added once."""
        N, D = self.N, self.D
        kern = self.ops.elbo_kernel_terms(self.a, self.b, self.nu, self.logdet_W, self.logdet_sigma_0, self.mm, D,
                                          self.a_0, self.b_0, self.nu_0)
        self.comm.sum_(kern)
        return kern[0] + self.ops.elbo_point_terms(self.c, D, -N * math.log(N - 1), self.a_0, self.b_0, self.nu_0)

    def log_pred_density(self, Y):
        """lakde/local_adaptive_kde.py:200-223 over the kernels of all ranks:
        log-mean of the per-rank mixtures, weighted by their kernel counts."""
        Y = Y.to(self.dtype)
        if self.n:
            S, nu = torch.empty_like(self.S), torch.empty_like(self.nu)
            self.ops.mstep(self.pat, self.r, self.X, self.lo, self.nu_0, S, nu, self.precision, self.err)
            U, logdet = torch.empty_like(self.U), torch.empty_like(self.logdet_W)
            info = torch.empty_like(self.info)
            self.ops.factor(S, self.W_inv_jitter, self.eps, self.sigma_0, self.nu_0_t, self.a, self.b, None, U, logdet,
                            None, info)
            v = self.ops.pred(self.X[self.lo : self.hi], U, nu, logdet, Y, self.precision, self.err) + math.log(self.n)
        else:
            v = torch.full((Y.size(0),), -math.inf, dtype=self.dtype, device=self.device)
        mx = v.clone()
        self.comm.max_(mx)
        safe = torch.where(torch.isfinite(mx), mx, torch.zeros_like(mx))
        se = torch.exp(v - safe)
        self.comm.sum_(se)
        return torch.where(torch.isfinite(mx), safe + torch.log(se), mx) - math.log(self.N)

    def responsibilities(self):
        """(kernel, point, r) of this rank's pairs, kernels in global numbering."""
        return self.pat.rows() + self.lo, self.pat.col.long(), self.r
