"""Kernels sharded over ranks (lakde_b200.shard), on CPU.

The per-shard arithmetic runs through a numpy stand-in built from the oracle
(the CUDA kernels need a GPU); the host logic under test is the sharding
itself: the kernel ranges, the per-shard pattern, the staged per-point
normaliser with its all-reduces between the stages, the ELBO and the
predictive-density reductions.  A world of two ``gloo`` ranks must reproduce
a world of one, which must reproduce the oracle's reference algorithm on the
same pair pattern.
"""

import datetime
import math
import os
import socket
import tempfile

import numpy as np
import pytest
import torch

from lakde_b200.shard import LocalComm, ShardedKNN, TorchComm, balanced_ranges, shard_pattern
from lakde_b200.sparse_util import PairPattern
from oracle import lakde_oracle as O

from .conftest import GOLDEN


class NumpyShardOps:
    """The per-shard steps of ShardedKNN restated with the oracle (CPU, any dtype)."""

    @staticmethod
    def _np(t):
        return t.detach().cpu().numpy()

    def prior(self, X, graph_rows, lo, jitter, eps):
        Xn = self._np(X)
        n = graph_rows.shape[0]
        sig = O.batched_knn_cov(Xn, Xn[lo : lo + n], self._np(graph_rows).astype(np.int64))
        L, jit = O.stabilized_cholesky(sig, self._np(jitter), eps=eps)
        if jit is not None:
            jitter.copy_(torch.from_numpy(np.asarray(jit)))
        sig = O._with_jitter(sig, self._np(jitter))
        return (torch.from_numpy(sig), torch.from_numpy(L), torch.from_numpy(O.chol_logdet(L)),
                torch.zeros((), dtype=torch.int32))

    def mstep(self, pat, r, X, lo, nu_0, S, nu, precision, err):
        Xn = self._np(X)
        n = S.shape[0]
        rowptr, col, rv = self._np(pat.rowptr), self._np(pat.col), self._np(r)
        S.copy_(torch.from_numpy(O.calc_W_inv(rowptr, col, rv, Xn[lo : lo + n], Xn)))
        nun = np.full(n, nu_0, dtype=Xn.dtype)
        np.add.at(nun, O._rows_of(rowptr), rv)
        nu.copy_(torch.from_numpy(nun))

    def factor(self, S, jitter, eps, P, nu_0, a, b, T, U, logdet, trace, info):
        Sn = self._np(S)
        e_tau = self._np(a) / self._np(b)
        A = (self._np(P) * (float(nu_0[0]) * e_tau)[:, None, None]).astype(Sn.dtype) + Sn
        L, jit = O.stabilized_cholesky(A, self._np(jitter), eps=eps)
        if jit is not None:
            jitter.copy_(torch.from_numpy(np.asarray(jit)))
        W = np.swapaxes(O.tril_inverse(L), -1, -2)
        U.copy_(torch.from_numpy(W))
        logdet.copy_(torch.from_numpy(O.chol_logdet(W)))
        info.zero_()
        if T is not None:
            trace.copy_(torch.from_numpy(O.chol_mm_trace(self._np(T), W)))

    def estep(self, pat, X, lo, U, nu, logdet, out, precision, err):
        lr = O.sparse_log_rho(self._np(pat.rowptr), self._np(pat.col), self._np(X), self._np(U), self._np(nu),
                              self._np(logdet), kernel_offset=lo)
        out.copy_(torch.from_numpy(lr))

    def normalise_stage(self, stage, pat, logrho, r, c, rsum, red, red2, mode, threshold):
        """The four stages of lakde_estep_normalise_stage over this rank's pairs."""
        col = self._np(pat.col).astype(np.int64)
        lr = self._np(logrho)
        dt = lr.dtype
        fi = np.finfo(dt)
        npts = c.numel()
        if stage == 0:
            mx = np.full(npts, -np.inf, dtype=dt)
            np.maximum.at(mx, col, lr)
            red.copy_(torch.from_numpy(mx))
        elif stage == 1:
            mx = self._np(red)
            ms = np.where(np.isfinite(mx), mx, 0).astype(dt)
            se = np.zeros(npts, dtype=dt)
            with np.errstate(invalid="ignore"):
                np.add.at(se, col, np.exp(lr - ms[col]).astype(dt))
            red2.copy_(torch.from_numpy(se))
        elif stage == 2:
            mx, se = self._np(red), self._np(red2)
            with np.errstate(divide="ignore"):
                lse = np.where(np.isfinite(mx), mx + np.log(se), -np.inf).astype(dt)
            cn, rs = self._np(c), self._np(rsum)
            if mode == 0:
                c_new = np.logaddexp(cn, lse).astype(dt)
            else:
                with np.errstate(divide="ignore"):
                    old = (np.log(rs) + cn).astype(dt)
                c_new = np.logaddexp(O.logsubexp(cn, old), lse).astype(dt)
            with np.errstate(invalid="ignore"):
                rv = np.exp(lr - c_new[col]).astype(dt)
            if threshold:
                rv = np.where(rv > threshold, rv, 0).astype(dt)
            sums = np.zeros(npts, dtype=dt)
            np.add.at(sums, col, rv)
            red.copy_(torch.from_numpy(c_new))
            red2.copy_(torch.from_numpy(sums))
        else:
            c_new, sums = self._np(red), np.maximum(self._np(red2), fi.eps).astype(dt)
            coeff = np.clip((1 / sums).astype(dt), fi.tiny, fi.max).astype(dt)
            with np.errstate(invalid="ignore"):
                rv = np.exp(lr - c_new[col]).astype(dt)
            if threshold:
                rv = np.where(rv > threshold, rv, 0).astype(dt)
            rv = (rv * coeff[col]).astype(dt)
            rs = np.zeros(npts, dtype=dt)
            np.add.at(rs, col, rv)
            r.copy_(torch.from_numpy(rv))
            c.copy_(torch.from_numpy((c_new + np.log(sums)).astype(dt)))
            rsum.copy_(torch.from_numpy(rs))

    def pred(self, Xk, U, nu, logdet, Y, precision=None, err=None):
        return torch.from_numpy(O.log_pred_density_from_factors(self._np(Xk), self._np(Y), self._np(U),
                                                                self._np(nu), self._np(logdet)))

    def elbo_kernel_terms(self, a, b, nu, logdet_W, logdet_sigma_0, mm, D, a_0, b_0, nu_0):
        """lakde/local_knn_kde.py:256-341, the per-kernel terms in float64 (torch on the host)."""
        from lakde_b200.linalg_util import lgamma, mvdigamma, mvlgamma

        f = lambda t: t.double()  # noqa: E731
        a, b, nu = f(a), f(b), f(nu)
        a_0, b_0, nu_0 = (torch.tensor(v, dtype=torch.float64) for v in (a_0, b_0, nu_0))
        log2 = math.log(2.0)
        e_tau = a / b
        e_log_tau = torch.digamma(a) - torch.log(b)
        e_logdet = mvdigamma(nu / 2, D) + D * log2 + f(logdet_W)
        p_tau = torch.sum(-lgamma(a_0) + a_0 * torch.log(b_0) + (a_0 - 1) * e_log_tau - b_0 * e_tau)
        q_tau = torch.sum(-lgamma(a) + a * torch.log(b) + (a - 1) * e_log_tau - b * e_tau)
        B_p = -nu_0 / 2 * (D * log2 - f(logdet_sigma_0) - D * e_log_tau - D * torch.log(nu_0)) - mvlgamma(
            nu_0 / 2, D)
        p_lam = torch.sum(B_p + (nu_0 - D - 1) * e_logdet / 2 - e_tau * nu_0 * f(mm) / 2)
        B_q = -nu / 2 * (f(logdet_W) + D * log2) - mvlgamma(nu / 2, D)
        q_lam = torch.sum(B_q + (nu - D - 1) * e_logdet / 2 - nu / 2 * D)
        return ((p_lam - q_lam) + (p_tau - q_tau)).reshape(1)

    def elbo_point_terms(self, c, D, tail, a_0=None, b_0=None, nu_0=None):
        return torch.sum(-D / 2 * math.log(2 * math.pi) + c.double()) + tail


class NumpyShardOpsFused(NumpyShardOps):
    """Adds the fused per-row pass of D <= 8 (lakde_vi_rows), restated with
    the oracle, so the sharded engine takes its one-pass branch."""

    def vi_rows(self, pat, r, X, lo, nu_0, a, b, b_0, jitter, eps, nu, logdet, info, logrho, P, T, mm):
        n, D = nu.shape[0], X.shape[1]
        S = torch.empty(n, D, D, dtype=X.dtype)
        U = torch.empty_like(S)
        trace = torch.empty(n, dtype=X.dtype)
        self.mstep(pat, r, X, lo, nu_0, S, nu, "fp32", None)
        # the factorisation reads E[tau] = a / b before b is updated
        self.factor(S, jitter, eps, P, torch.tensor([nu_0], dtype=X.dtype), a, b, T, U, logdet, trace, info)
        mm.copy_(nu * trace)
        b.copy_(b_0 + nu_0 * mm / 2)
        self.estep(pat, X, lo, U, nu, logdet, logrho, "fp32", None)


ITERS, THR = 4, 1e-4


def knn_pattern(graph):
    """The kNN pair pattern (graph[m, k], m) built on the host (numpy)."""
    graph = np.asarray(graph)
    N, Kn = graph.shape
    kern = graph.reshape(-1).astype(np.int64)
    point = np.repeat(np.arange(N), Kn)
    rank = np.tile(np.arange(Kn, dtype=np.int32), N)
    order = np.argsort(kern * N + point, kind="stable")
    kern, point, rank = kern[order], point[order], rank[order]
    rowptr = O.ind2ptr(kern, N)
    pos = np.argsort(point * N + kern, kind="stable")
    cptr = O.ind2ptr(point[pos], N)
    t = torch.from_numpy
    return PairPattern(t(rowptr), t(point.astype(np.int32)), t(cptr), t(pos.astype(np.int32)), N, N, t(rank))


def _fit(world, rank, port, outdir, fused=False):
    torch.set_num_threads(1)
    comm = LocalComm()
    if world > 1:
        import torch.distributed as dist

        dist.init_process_group("gloo", rank=rank, world_size=world, init_method=f"tcp://127.0.0.1:{port}",
                                timeout=datetime.timedelta(seconds=120))
        comm = TorchComm()
    g = np.load(os.path.join(GOLDEN, "knn_small_f64_bN.npz"))
    X = torch.tensor(g["X"], dtype=torch.float64)
    Y = torch.tensor(g["Y"], dtype=torch.float64)
    graph = torch.tensor(g["knn_graph"])
    D = X.shape[1]
    pattern = knn_pattern(g["knn_graph"])
    eng = ShardedKNN(X, graph, pattern, nu_0=D, a_0=1e-6, b_0=1e-6, threshold=THR, init_k=graph.shape[1],
                     comm=comm, ops=NumpyShardOpsFused() if fused else NumpyShardOps())
    assert D <= 8  # the fused per-row branch is the D <= 8 step
    eng.init_summaries()
    elbo = []
    for _ in range(ITERS):
        eng.step()
        elbo.append(float(eng.compute_elbo()))
    eng.check_errors()
    lpd = eng.log_pred_density(Y)
    k, m, r = eng.responsibilities()
    np.savez(os.path.join(outdir, f"w{world}_r{rank}_f{int(fused)}.npz"), elbo=np.array(elbo), c=eng.c.numpy(),
             rsum=eng.rsum.numpy(), lpd=lpd.numpy(), k=k.numpy(), m=m.numpy(), r=r.numpy(), lo=eng.lo, hi=eng.hi)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


def _spawned(rank, world, port, outdir, fused):
    _fit(world, rank, port, outdir, fused)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.fixture(scope="module", params=[False, True], ids=["four-pass", "fused-rows"])
def runs(request):
    """World 1 and a gloo world of 2, through the four-pass step or the fused
    per-row step (NumpyShardOpsFused.vi_rows)."""
    import torch.multiprocessing as mp

    fused = request.param
    outdir = tempfile.mkdtemp(prefix="lakde_shard_")
    _fit(1, 0, 0, outdir, fused)
    mp.spawn(_spawned, args=(2, _free_port(), outdir, fused), nprocs=2, join=True)
    load = lambda w, r: dict(np.load(os.path.join(outdir, f"w{w}_r{r}_f{int(fused)}.npz")))  # noqa: E731
    return load(1, 0), [load(2, 0), load(2, 1)]


def test_balanced_ranges_cover_all_kernels():
    rowptr = torch.tensor(np.concatenate([[0], np.cumsum(np.random.default_rng(0).integers(0, 50, 1001))]))
    for world in (1, 2, 3, 8):
        rs = balanced_ranges(rowptr, world)
        assert rs[0][0] == 0 and rs[-1][1] == 1001
        assert all(a[1] == b[0] for a, b in zip(rs, rs[1:]))
        sizes = [int(rowptr[h] - rowptr[lo]) for lo, h in rs]
        assert max(sizes) - min(sizes) <= 2 * 50


def test_shard_patterns_partition_the_pairs():
    g = np.load(os.path.join(GOLDEN, "knn_small_f64_bN.npz"))
    pattern = knn_pattern(g["knn_graph"])
    keys = []
    for lo, hi in balanced_ranges(pattern.rowptr, 3):
        p = shard_pattern(pattern, lo, hi)
        assert p.n_kernels == hi - lo and p.n_points == pattern.n_points
        k = p.rows() + lo
        keys.append(k * pattern.n_points + p.col.long())
        # point-major view of the shard: every local pair once, grouped by point
        pts = p.col.long()[p.pos.long()]
        assert torch.equal(pts, torch.sort(pts).values)
        assert torch.equal(torch.sort(p.pos.long()).values, torch.arange(p.nnz))
    allk = torch.cat(keys)
    assert torch.equal(allk, pattern.rows() * pattern.n_points + pattern.col.long())


def test_one_rank_matches_the_restricted_oracle(runs):
    one, _ = runs
    g = np.load(os.path.join(GOLDEN, "knn_small_f64_bN.npz"))
    X, graph = g["X"].astype(np.float64), g["knn_graph"]
    N = len(X)
    mask = np.zeros((N, N), dtype=bool)
    mask[graph.reshape(-1), np.repeat(np.arange(N), graph.shape[1])] = True
    ora = O.KNNKDEOracle(k=graph, block_size=N, candidates=mask)
    el = []
    ora.fit(X, iterations=ITERS, threshold=THR, callback=lambda mm, XX: el.append(mm.compute_elbo(XX)))
    np.testing.assert_allclose(one["elbo"], el, rtol=1e-10)
    np.testing.assert_allclose(one["c"], ora.rnm_log_consts, atol=1e-9)
    np.testing.assert_allclose(one["lpd"], ora.log_pred_density(X, g["Y"].astype(np.float64)), atol=1e-9)


def test_two_ranks_match_one(runs):
    one, two = runs
    # the ranks split the kernels and agree on every per-point quantity
    assert two[0]["lo"] == 0 and two[0]["hi"] == two[1]["lo"] and two[1]["hi"] == len(one["c"])
    np.testing.assert_array_equal(two[0]["c"], two[1]["c"])
    np.testing.assert_array_equal(two[0]["rsum"], two[1]["rsum"])
    np.testing.assert_array_equal(two[0]["elbo"], two[1]["elbo"])
    np.testing.assert_array_equal(two[0]["lpd"], two[1]["lpd"])
    np.testing.assert_allclose(two[0]["c"], one["c"], rtol=0, atol=1e-12)
    np.testing.assert_allclose(two[0]["rsum"], one["rsum"], rtol=1e-12)
    np.testing.assert_allclose(two[0]["elbo"], one["elbo"], rtol=1e-13)
    np.testing.assert_allclose(two[0]["lpd"], one["lpd"], rtol=0, atol=1e-12)
    r2 = np.concatenate([two[0]["r"], two[1]["r"]])
    k2 = np.concatenate([two[0]["k"], two[1]["k"]])
    m2 = np.concatenate([two[0]["m"], two[1]["m"]])
    np.testing.assert_array_equal(k2, one["k"])
    np.testing.assert_array_equal(m2, one["m"])
    np.testing.assert_allclose(r2, one["r"], rtol=1e-12, atol=1e-15)
