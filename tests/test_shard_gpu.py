"""The sharded path's GPU pieces with one device: the staged per-point pass
equals the single-kernel pass, the tensor-core kernels honour a kernel
offset, and a world of one reproduces the unsharded engine.  (Several GPUs
are covered on CPU by tests/test_shard.py.)"""

import numpy as np
import pytest
import torch

from oracle import lakde_oracle as O

pytestmark = pytest.mark.gpu
DEV = "cuda"


def t(a, dtype=None):
    out = torch.tensor(np.asarray(a), device=DEV)
    return out if dtype is None else out.to(dtype)


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
@pytest.mark.parametrize("mode", [0, 1])
def test_staged_normaliser_equals_single_pass(dtype, mode):
    from lakde_b200 import kernels as K
    from lakde_b200.sparse_util import PairPattern

    rng = np.random.default_rng(7)
    N = 2000
    counts = rng.integers(1, 300, N)  # rows above and below the 128-pair register path
    kern = np.repeat(np.arange(N), counts)
    point = rng.integers(0, N, kern.size)
    keep = np.unique(kern * N + point, return_index=True)[1]
    p = PairPattern.from_pairs(t(kern[keep]), t(point[keep]), N, N)
    logrho = t(rng.standard_normal(p.nnz) * 3 - 5, dtype)
    c0 = t(rng.standard_normal(N) * 0.1 - 1, dtype)
    rs0 = t(rng.uniform(0.5, 1.5, N), dtype)
    r1, c1, rs1 = torch.zeros_like(logrho), c0.clone(), rs0.clone()
    K.estep_normalise(p.cptr, p.pos, logrho, r1, c1, rs1, mode, 1e-4)
    r2, c2, rs2 = torch.zeros_like(logrho), c0.clone(), rs0.clone()
    red, red2 = torch.empty_like(c0), torch.empty_like(c0)
    for stage in range(4):
        K.estep_normalise_stage(stage, p.cptr, p.pos, logrho, r2, c2, rs2, red, red2, mode, 1e-4)
    torch.testing.assert_close(r2, r1, rtol=0, atol=0)
    torch.testing.assert_close(c2, c1, rtol=0, atol=0)
    torch.testing.assert_close(rs2, rs1, rtol=0, atol=0)


@pytest.mark.parametrize("D", [21, 63])
def test_tc_kernels_honour_the_kernel_offset(D):
    from lakde_b200 import kernels as K

    rng = np.random.default_rng(D)
    N, k = 400, 30
    X = (rng.standard_normal((N, D)) * 2 + 5).astype(np.float32)
    graph = O.knn_graph(X, k)
    ((rows, cols),) = O.knn_pattern(graph)
    rowptr = O.ind2ptr(rows, N)
    r = rng.uniform(0, 1, cols.size).astype(np.float32)
    W = np.triu(rng.standard_normal((N, D, D)) / np.sqrt(D)).astype(np.float32)
    W[:, np.arange(D), np.arange(D)] = np.abs(W[:, np.arange(D), np.arange(D)]) + 1
    nu = rng.uniform(D + 1, D + 10, N).astype(np.float32)
    logdet = O.chol_logdet(W).astype(np.float32)
    err = torch.zeros(1, dtype=torch.int32, device=DEV)
    S, nuo = K.mstep_tc(t(rowptr), t(cols, torch.int32), t(r), t(X), D + 1.0, err)
    Wc = K.pack_w_cores(t(W))
    lr = K.estep_tc(t(rowptr), t(cols, torch.int32), t(X), Wc, t(nu), t(logdet), err)
    lo, hi = 123, 301
    p0, p1 = rowptr[lo], rowptr[hi]
    rp = rowptr[lo : hi + 1] - p0
    S2, nu2 = K.mstep_tc(t(rp), t(cols[p0:p1], torch.int32), t(r[p0:p1]), t(X), D + 1.0, err, kernel_offset=lo)
    lr2 = K.estep_tc(t(rp), t(cols[p0:p1], torch.int32), t(X), Wc[lo:hi].contiguous(), t(nu[lo:hi]),
                     t(logdet[lo:hi]), err, kernel_offset=lo)
    assert int(err) == 0
    torch.testing.assert_close(S2, S[lo:hi], rtol=0, atol=0)
    torch.testing.assert_close(nu2, nuo[lo:hi], rtol=0, atol=0)
    torch.testing.assert_close(lr2, lr[p0:p1], rtol=0, atol=0)
    # the self pairs of the offset rows are -inf
    self_pair = cols[p0:p1] == np.repeat(np.arange(lo, hi), np.diff(rp))
    assert torch.isneginf(lr2[t(self_pair)]).all()


@pytest.mark.parametrize("D", [3, 5, 8])
def test_fused_row_kernels_honour_the_kernel_offset(D):
    """lakde_vi_rows (D <= 8) on a shard's rows (kernel_offset) gives the rows
    of the full launch bit for bit."""
    from lakde_b200 import kernels as K

    rng = np.random.default_rng(D + 1)
    N, k = 400, 24
    X = (rng.standard_normal((N, D)) * 2 + 5).astype(np.float32)
    graph = O.knn_graph(X, k)
    ((rows, cols),) = O.knn_pattern(graph)
    rowptr = O.ind2ptr(rows, N)
    r = rng.uniform(0, 1, cols.size).astype(np.float32)
    A = rng.standard_normal((N, D, D + 3))
    P = (A @ np.swapaxes(A, 1, 2) / (D + 3) + 0.1 * np.eye(D)).astype(np.float32)
    T = np.linalg.cholesky(P.astype(np.float64)).astype(np.float32)
    a = np.full(N, 1.0 + D / 2, np.float32)
    b = rng.uniform(0.5, 2.0, N).astype(np.float32)

    def run(lo, hi):
        p0, p1 = rowptr[lo], rowptr[hi]
        n = hi - lo
        out = dict(b=t(b[lo:hi].copy()), jitter=t(np.zeros(n, np.float32)), nu=t(np.zeros(n, np.float32)),
                   logdet=t(np.zeros(n, np.float32)), info=t(np.zeros(n, np.int32)),
                   logrho=t(np.zeros(p1 - p0, np.float32)), mm=t(np.zeros(n, np.float32)))
        K.vi_rows(t(rowptr[lo:hi + 1] - p0), t(cols[p0:p1], torch.int32), t(r[p0:p1]), t(X), float(D), t(a[lo:hi]),
                  out["b"], 1e-6, out["jitter"], 1.2e-7, out["nu"], out["logdet"], out["info"], out["logrho"],
                  P=t(P[lo:hi]), T=t(T[lo:hi]), mm=out["mm"], kernel_offset=lo)
        return out

    full = run(0, N)
    lo, hi = 123, 301
    part = run(lo, hi)
    p0, p1 = rowptr[lo], rowptr[hi]
    for key in ("b", "jitter", "nu", "logdet", "info", "mm"):
        torch.testing.assert_close(part[key], full[key][lo:hi], rtol=0, atol=0)
    torch.testing.assert_close(part["logrho"], full["logrho"][p0:p1], rtol=0, atol=0)
    self_pair = cols[p0:p1] == np.repeat(np.arange(lo, hi), np.diff(rowptr[lo:hi + 1]))
    assert torch.isneginf(part["logrho"][t(self_pair)]).all()


@pytest.mark.parametrize("precision,d", [("fp32", 13), ("mixed", 13), ("fp32", 5)])
def test_world_of_one_matches_the_fused_engine(precision, d):
    from lakde_b200.engine import FusedKNN
    from lakde_b200.shard import ShardedKNN
    from lakde_b200.sparse_util import PairPattern
    from lakde_b200.synthetic import heavy_tail_mixture
    from lakde_b200.utils import compute_knn_graph

    Xn, Yn = heavy_tail_mixture(seed=2, n_train=3000, n_test=200, d=d)
    X, Y = t(Xn.astype(np.float32)), t(Yn.astype(np.float32))
    graph = compute_knn_graph(X, 16)
    pattern = PairPattern.from_knn_graph(graph)
    tiny = torch.tensor(1e-6, device=DEV)
    kw = dict(nu_0=float(d), a_0=tiny, b_0=tiny, threshold=5e-4, init_k=16, precision=precision)
    ref = FusedKNN(X, graph, pattern, **kw)
    sh = ShardedKNN(X, graph, pattern, **kw)
    ref.init_summaries()
    sh.init_summaries()
    for _ in range(3):
        ref.step()
        sh.step()
    ref.check_errors()
    sh.check_errors()
    torch.testing.assert_close(sh.c, ref.c, rtol=0, atol=0)
    torch.testing.assert_close(sh.r, ref.r, rtol=0, atol=0)
    assert abs(float(sh.compute_elbo()) - float(ref.compute_elbo())) <= 1e-9 * abs(float(ref.compute_elbo()))
    torch.testing.assert_close(sh.log_pred_density(Y), ref.log_pred_density(Y), rtol=0, atol=2e-5)


def test_elbo_parts_over_two_kernel_ranges_sum_to_the_whole():
    """The sharded ELBO: the kernel terms of two kernel ranges (two ranks) plus
    the point terms once equal lakde_knn_elbo over all kernels and points."""
    from lakde_b200 import kernels as K

    rng = np.random.default_rng(7)
    N, D = 1000, 13
    a = t(rng.uniform(5, 9, N))
    b = t(rng.uniform(0.5, 2, N))
    nu = t(rng.uniform(D + 1, D + 40, N))
    ldw = t(rng.normal(0, 3, N))
    lds0 = t(rng.normal(-5, 2, N))
    mm = t(rng.uniform(1, 50, N))
    c = t(rng.normal(-2, 1, N))
    a_0, b_0, nu_0 = 1e-6, 1e-6, float(D)
    whole = float(K.knn_elbo(a, b, nu, ldw, lds0, mm, c, a_0, b_0, nu_0, D))
    cut = 377
    parts = 0.0
    for lo, hi in ((0, cut), (cut, N)):
        parts += float(K.knn_elbo_parts(D, a_0, b_0, nu_0, a=a[lo:hi], b=b[lo:hi], nu=nu[lo:hi],
                                        logdet_W=ldw[lo:hi], logdet_sigma_0=lds0[lo:hi], mm=mm[lo:hi]))
    parts += float(K.knn_elbo_parts(D, a_0, b_0, nu_0, c=c, tail=-N * np.log(N - 1)))
    assert abs(parts - whole) <= 1e-12 * abs(whole)
    # a points-only call does not depend on the kernel hyper-parameters
    p1 = float(K.knn_elbo_parts(D, a_0, b_0, nu_0, c=c))
    p2 = float(K.knn_elbo_parts(D, 0.0, 0.0, 0.0, c=c))
    assert p1 == p2 and np.isfinite(p2)
