"""Parity of the CUDA ops (through the C ABI) with the golden vectors of the
reference and with the oracle."""

import os

import numpy as np
import pytest
import torch

from oracle import lakde_oracle as O

from .conftest import GOLDEN

pytestmark = pytest.mark.gpu

DEV = "cuda"


@pytest.fixture(scope="module")
def K():
    from lakde_b200 import kernels

    return kernels


@pytest.fixture(scope="module")
def ops():
    return np.load(os.path.join(GOLDEN, "ops.npz"))


def t(a, dtype=None):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV, dtype=dtype)


def rand_upper(rng, N, D, dtype):
    W = np.triu(rng.standard_normal((N, D, D)))
    W[:, np.arange(D), np.arange(D)] = np.abs(W[:, np.arange(D), np.arange(D)]) + 0.5
    return W.astype(dtype)


# ----------------------------------------------------------------- quad form
@pytest.mark.parametrize("dt", ["f32", "f64"])
@pytest.mark.parametrize("D", [1, 2, 5, 8, 17, 33])
def test_quad_form_golden(K, ops, dt, D):
    k = f"quad_{dt}_d{D}"
    Q = K.chol_quad_form(t(ops[k + "_W"]), t(ops[k + "_Xn"]), t(ops[k + "_Xm"]))
    rtol = 1e-5 if dt == "f32" else 1e-12
    np.testing.assert_allclose(Q.cpu().numpy(), ops[k + "_Q"], rtol=rtol, atol=rtol)


@pytest.mark.parametrize("D", [2, 8, 21, 43, 63, 64])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_quad_form_random_strided(K, D, dtype):
    rng = np.random.default_rng(D)
    N, M = 37, 301
    W = (rand_upper(rng, N, D, dtype) / np.sqrt(D)).astype(dtype)
    Xn = rng.standard_normal((N, D)).astype(dtype)
    Xm = rng.standard_normal((M, D)).astype(dtype)
    ref = O.chol_quad_form(W.astype(np.float64), Xn.astype(np.float64), Xm.astype(np.float64))
    # strided inputs and a transposed output, as the reference op accepts
    Wt = t(np.ascontiguousarray(W.transpose(0, 2, 1))).transpose(1, 2)
    Xnt = t(np.ascontiguousarray(Xn.T)).T
    out = torch.empty(M, N, dtype=Wt.dtype, device=DEV).T
    torch.ops.lakde.chol_quad_form_cuda(Wt, Xnt, t(Xm), out)
    rtol = 2e-5 if dtype == np.float32 else 1e-11
    np.testing.assert_allclose(out.cpu().numpy(), ref, rtol=rtol, atol=rtol * ref.max())


def test_quad_form_rejects_large_d_and_cpu(K):
    W = torch.zeros(2, 65, 65, device=DEV)
    X = torch.zeros(2, 65, device=DEV)
    with pytest.raises(RuntimeError, match="exceeds"):
        K.chol_quad_form(W, X, X)
    with pytest.raises(RuntimeError):
        K.chol_quad_form(W.cpu(), X.cpu(), X.cpu())


# ------------------------------------------------------------- scatter (M-step)
@pytest.mark.parametrize("dt", ["f32", "f64"])
@pytest.mark.parametrize("D", [1, 3, 7, 16])
@pytest.mark.parametrize("idx", [(torch.int64, torch.int64), (torch.int32, torch.int32), (torch.int32, torch.int64),
                                 (torch.int64, torch.int32)])
def test_W_inv_golden(K, ops, dt, D, idx):
    k = f"winv_{dt}_d{D}"
    rowptr, col, value, Xn, Xm = (ops[f"{k}_{n}"] for n in ("rowptr", "col", "value", "Xn", "Xm"))
    S = K.calc_W_inv(t(rowptr, idx[0]), t(col, idx[1]), t(value), t(Xn), t(Xm))
    rtol = 1e-5 if dt == "f32" else 1e-12
    np.testing.assert_allclose(S.cpu().numpy(), ops[k + "_S"], rtol=rtol, atol=rtol)


@pytest.mark.parametrize("D", [2, 8, 21, 43, 63])
def test_W_inv_random(K, D):
    rng = np.random.default_rng(100 + D)
    N, M = 50, 400
    counts = rng.integers(0, 150, size=N)
    counts[[3, 17]] = 0
    counts[5] = 700  # a long row (several chunks)
    rowptr = np.concatenate([[0], np.cumsum(counts)])
    col = rng.integers(0, M, size=rowptr[-1])
    val = rng.uniform(0, 1, size=rowptr[-1]).astype(np.float32)
    Xn = rng.standard_normal((N, D)).astype(np.float32)
    Xm = rng.standard_normal((M, D)).astype(np.float32)
    ref = O.calc_W_inv(rowptr, col, val.astype(np.float64), Xn.astype(np.float64), Xm.astype(np.float64))
    S = K.calc_W_inv(t(rowptr), t(col, torch.int32), t(val), t(Xn), t(Xm)).cpu().numpy()
    np.testing.assert_allclose(S, ref, rtol=1e-4, atol=1e-4 * np.abs(ref).max())
    np.testing.assert_array_equal(S, np.swapaxes(S, 1, 2))


@pytest.mark.parametrize("D", [3, 40])
def test_W_inv_invalid_column_gives_nan_row(K, D):
    rowptr = torch.tensor([0, 2, 4], device=DEV)
    col = torch.tensor([0, 1, 1, 99], device=DEV)
    val = torch.ones(4, device=DEV)
    X = torch.randn(3, D, device=DEV)
    S = K.calc_W_inv(rowptr, col, val, X[:2].contiguous(), X)
    assert torch.isfinite(S[0]).all()
    assert torch.isnan(S[1]).all()


# ------------------------------------------------------------------- ind2ptr
@pytest.mark.parametrize("din,dout", [(torch.int32, torch.int32), (torch.int64, torch.int64),
                                      (torch.int32, torch.int64)])
def test_ind2ptr(K, ops, din, dout):
    row = t(ops["ind2ptr_row"], din)
    M = int(ops["ind2ptr_M"])
    out = torch.empty(M + 1, dtype=dout, device=DEV)
    torch.ops.lakde.ind2ptr_cuda(row, M, out)
    np.testing.assert_array_equal(out.cpu().numpy(), ops["ind2ptr_out"])
    empty = K.ind2ptr(torch.zeros(0, dtype=din, device=DEV), 7)
    assert empty.cpu().tolist() == [0] * 8


def test_ind2ptr_large(K):
    rng = np.random.default_rng(0)
    row = np.sort(rng.integers(0, 100_000, size=3_000_000))
    out = K.ind2ptr(t(row), 100_000)
    np.testing.assert_array_equal(out.cpu().numpy(), O.ind2ptr(row, 100_000))


# ---------------------------------------------------------- posterior factor
@pytest.mark.parametrize("dt", ["f32", "f64"])
def test_factor_jitter_ladder_golden(K, ops, dt):
    X = ops[f"chol_{dt}_X"]
    jit = t(np.zeros(len(X), X.dtype))
    W, logdet, info, L, _ = K.posterior_factor(t(X), jit, np.finfo(X.dtype).eps, want_L=True)
    assert (info.cpu().numpy() == 0).all()
    jit = jit.cpu().numpy()
    ref = ops[f"chol_{dt}_jitter"]
    np.testing.assert_array_equal(jit[:4], 0)
    np.testing.assert_array_equal(jit == 0, ref == 0)
    eps = np.finfo(X.dtype).eps
    nz = jit != 0
    k = np.log2(jit[nz] / eps + 1)
    np.testing.assert_allclose(k, np.round(k), atol=1e-9)
    if dt == "f64":
        assert jit[6] == ref[6]
    # the factor of the jittered matrix: L L^T reproduces X + jitter I (the
    # rank-deficient ones only up to rounding), and the full-rank ones match LAPACK
    Xj = X.astype(np.float64) + np.eye(X.shape[1]) * jit[:, None, None]
    Lg = L.cpu().numpy().astype(np.float64)
    recon = Lg @ np.swapaxes(Lg, 1, 2)
    scale = np.abs(Xj).max(axis=(1, 2))[:, None, None]
    tol = 64 * np.finfo(X.dtype).eps * X.shape[1]
    assert (np.abs(recon - Xj) <= tol * scale).all()
    Lref = np.linalg.cholesky(Xj[:4])
    np.testing.assert_allclose(Lg[:4], Lref, rtol=1e-4, atol=1e-5 * np.abs(Lref).max())


def spd(rng, N, D, cond=1e3):
    A = rng.standard_normal((N, D, D))
    Q, _ = np.linalg.qr(A)
    ev = np.exp(rng.uniform(0, np.log(cond), size=(N, D)))
    return np.einsum("nij,nj,nkj->nik", Q, ev, Q)


@pytest.mark.parametrize("D", [1, 2, 5, 8, 13, 21, 43, 63])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_factor_random(K, D, dtype):
    rng = np.random.default_rng(D)
    N = 67
    S = spd(rng, N, D).astype(dtype)
    P = spd(rng, N, D).astype(dtype)
    a = rng.uniform(1, 3, N).astype(dtype)
    b = rng.uniform(1, 3, N).astype(dtype)
    nu0 = np.array(D + 1.5, dtype=dtype)
    Tm = np.tril(rng.standard_normal((N, D, D))).astype(dtype)
    jit = t(np.zeros(N, dtype))
    W, logdet, info, L, trace = K.posterior_factor(t(S), jit, np.finfo(dtype).eps, P=t(P), nu_0=t(nu0), a=t(a),
                                                   b=t(b), T=t(Tm), want_L=True)
    assert (info.cpu().numpy() == 0).all() and (jit.cpu().numpy() == 0).all()
    A = (P.astype(np.float64) * (nu0 * (a / b)).astype(np.float64)[:, None, None]) + S
    Lr = np.linalg.cholesky(A)
    Ur = np.swapaxes(np.linalg.inv(Lr), 1, 2)
    rtol = 1e-4 if dtype == np.float32 else 1e-9
    np.testing.assert_allclose(W.cpu().numpy(), Ur, rtol=rtol, atol=rtol * np.abs(Ur).max())
    np.testing.assert_allclose(L.cpu().numpy(), Lr, rtol=rtol, atol=rtol * np.abs(Lr).max())
    np.testing.assert_allclose(logdet.cpu().numpy(), O.chol_logdet(Ur), rtol=rtol, atol=rtol * 10)
    np.testing.assert_allclose(trace.cpu().numpy(), O.chol_mm_trace(Tm.astype(np.float64), Ur), rtol=10 * rtol)
    # declaring T lower triangular skips its upper part: same results, and
    # garbage above the diagonal is not read
    Tg = Tm + np.triu(rng.standard_normal((N, D, D)), 1).astype(dtype)
    jit2 = t(np.zeros(N, dtype))
    W2, logdet2, info2, _, trace2 = K.posterior_factor(t(S), jit2, np.finfo(dtype).eps, P=t(P), nu_0=t(nu0),
                                                       a=t(a), b=t(b), T=t(Tg), T_lower=True)
    torch.testing.assert_close(W2, W, rtol=0, atol=0)
    torch.testing.assert_close(logdet2, logdet, rtol=0, atol=0)
    np.testing.assert_allclose(trace2.cpu().numpy(), trace.cpu().numpy(), rtol=1e-12 if dtype == np.float64 else 1e-5)


def test_factor_shared_prior_and_failure(K):
    rng = np.random.default_rng(3)
    D, N = 6, 10
    S = spd(rng, N, D)
    P = spd(rng, 1, D)[0]
    jit = t(np.zeros(N))
    W, logdet, info, _, trace = K.posterior_factor(t(S), jit, 2.2e-16, P=t(P), T=t(P))
    A = S + P
    Ur = np.swapaxes(np.linalg.inv(np.linalg.cholesky(A)), 1, 2)
    np.testing.assert_allclose(W.cpu().numpy(), Ur, rtol=1e-9, atol=1e-12)
    # a matrix no ladder rung repairs: info = -1 and NaN outputs
    bad = -np.eye(D)[None].repeat(2, 0) * 1e3
    jit = t(np.zeros(2))
    W, logdet, info, _, _ = K.posterior_factor(t(bad), jit, 2.2e-16)
    assert (info.cpu().numpy() == -1).all()
    assert torch.isnan(W).all() and torch.isnan(logdet).all()


# ----------------------------------------------------------- sparse E-step
def small_problem(rng, N=300, D=5, K=12, dtype=np.float32):
    X = rng.standard_normal((N, D)).astype(dtype)
    graph = O.knn_graph(X, K)
    (pat,) = O.knn_pattern(graph)
    rows, cols = pat
    rowptr = O.ind2ptr(rows, N)
    W = rand_upper(rng, N, D, dtype) * 2
    nu = rng.uniform(D + 1, D + 10, N).astype(dtype)
    logdet = O.chol_logdet(W).astype(dtype)
    return X, rowptr, cols, W, nu, logdet


@pytest.mark.parametrize("D", [2, 5, 21])
def test_estep_logrho_and_normalise(K, D):
    rng = np.random.default_rng(D)
    X, rowptr, cols, W, nu, logdet = small_problem(rng, D=D)
    N = len(X)
    lr = K.estep_logrho(t(rowptr), t(cols, torch.int32), t(X), t(W), t(nu), t(logdet)).cpu().numpy()
    ref = O.sparse_log_rho(rowptr, cols, X, W, nu, logdet)
    np.testing.assert_allclose(lr, ref, rtol=1e-4, atol=1e-4 * np.abs(ref).max())
    # point-major view
    order = np.argsort(cols, kind="stable")
    cptr = O.ind2ptr(cols[order], N)
    c0 = np.full(N, -np.inf, np.float32)
    rs0 = np.zeros(N, np.float32)
    for mode, thr in ((0, 0.0), (1, 1e-3)):
        lr_t = t(ref)
        r = torch.zeros_like(lr_t)
        c = t(c0.copy())
        rs = t(rs0.copy())
        K.estep_normalise(t(cptr), t(order), lr_t, r, c, rs, mode, thr)
        r_ref, c_ref, rs_ref = O.sparse_normalise(cols, ref, c0, rs0, N, mode, thr)
        np.testing.assert_allclose(r.cpu().numpy(), r_ref, rtol=1e-5, atol=1e-7)
        np.testing.assert_allclose(c.cpu().numpy(), c_ref, rtol=1e-6, atol=1e-5)
        np.testing.assert_allclose(rs.cpu().numpy(), rs_ref, rtol=1e-5)
        c0, rs0 = c_ref, rs_ref


def test_estep_self_pairs_are_excluded(K):
    rng = np.random.default_rng(9)
    X = rng.standard_normal((50, 3)).astype(np.float32)
    graph = O.knn_graph(X, 5, include_self=True)
    ((rows, cols),) = O.knn_pattern(graph)
    W = rand_upper(rng, 50, 3, np.float32)
    nu = np.full(50, 6, np.float32)
    logdet = O.chol_logdet(W).astype(np.float32)
    lr = K.estep_logrho(t(O.ind2ptr(rows, 50)), t(cols), t(X), t(W), t(nu), t(logdet)).cpu().numpy()
    assert np.all(np.isneginf(lr[rows == cols]))
    assert np.all(np.isfinite(lr[rows != cols]))


# ---------------------------------------------------------- predictive density
@pytest.mark.parametrize("D", [2, 8, 21, 43, 63])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_log_pred_density(K, D, dtype):
    rng = np.random.default_rng(D)
    N, Nq = 1500, 700
    X = rng.standard_normal((N, D)).astype(dtype)
    Y = rng.standard_normal((Nq, D)).astype(dtype)
    W = (rand_upper(rng, N, D, dtype) / np.sqrt(D)).astype(dtype)
    nu = rng.uniform(D + 1, D + 30, N).astype(dtype)
    logdet = O.chol_logdet(W).astype(dtype)
    lc = K.pred_coeff(t(nu), t(logdet), D)
    out = K.log_pred_density(t(X), t(W), t(nu), lc, t(Y)).cpu().numpy()
    ref = O.log_pred_density_from_factors(X.astype(np.float64), Y.astype(np.float64), W.astype(np.float64),
                                          nu.astype(np.float64), logdet.astype(np.float64))
    atol = 2e-4 if dtype == np.float32 else 1e-9
    np.testing.assert_allclose(out, ref, rtol=0, atol=atol * max(1, D / 8))


# ------------------------------------------------------- fused per-row pass
@pytest.mark.parametrize("D,dtype", [(2, np.float32), (5, np.float32), (8, np.float32), (2, np.float64),
                                     (5, np.float64), (8, np.float64)])
def test_vi_rows_matches_unfused_composition(K, D, dtype):
    rng = np.random.default_rng(10 + D)
    N = 400
    X = rng.standard_normal((N, D)).astype(dtype)
    graph = O.knn_graph(X, 12 if D <= 8 else 40)
    ((rows, cols),) = O.knn_pattern(graph)
    rowptr = O.ind2ptr(rows, N)
    r = rng.uniform(0.01, 1, size=len(cols)).astype(dtype)
    P = spd(rng, N, D, cond=10).astype(dtype) * 0.1
    # rows 0..6: no prior and a single weighted pair, so S is rank one and
    # the jitter ladder has to run
    P[:7] = 0
    for n in range(7):
        r[rowptr[n] + 1 : rowptr[n + 1]] = 0
    Tm = np.linalg.cholesky(P.astype(np.float64) + np.eye(D) * 1e-3).astype(dtype)
    a = rng.uniform(2, 4, N).astype(dtype)
    b = rng.uniform(1, 3, N).astype(dtype)
    nu0, b0 = D + 0.5, 1e-6
    eps = np.finfo(dtype).eps
    # unfused reference composition
    rp, cl, rr, Xt = t(rowptr), t(cols, torch.int32), t(r), t(X)
    S, nu = K.mstep(rp, cl, rr, Xt, nu0)
    jit1 = torch.zeros(N, dtype=Xt.dtype, device=DEV)
    W, logdet, info, _, trace = K.posterior_factor(S, jit1, eps, P=t(P), nu_0=torch.tensor(nu0, device=DEV),
                                                   a=t(a), b=t(b), T=t(Tm))
    lr_ref = K.estep_logrho(rp, cl, Xt, W, nu, logdet)
    mm_ref = nu * trace
    b_ref = b0 + nu0 * mm_ref / 2
    # fused
    bt = t(b)
    jit2 = torch.zeros_like(jit1)
    nu2, ld2, mm2 = torch.empty_like(nu), torch.empty_like(nu), torch.empty_like(nu)
    info2 = torch.empty(N, dtype=torch.int32, device=DEV)
    lr2 = torch.empty_like(lr_ref)
    pattern_order = torch.argsort(torch.tensor(np.diff(rowptr), device=DEV), descending=True).to(torch.int32)
    K.vi_rows(rp, cl, rr, Xt, nu0, t(a), bt, b0, jit2, eps, nu2, ld2, info2, lr2, P=t(P), T=t(Tm),
              order=pattern_order, mm=mm2)
    assert (info2 == 0).all() and (info == 0).all()
    # rank-one rows mostly need the ladder (a 2 x 2 one may factor by rounding)
    assert (jit1[:7] > 0).any()
    torch.testing.assert_close(jit2, jit1, rtol=0, atol=0)
    rtol = 1e-4 if dtype == np.float32 else 1e-9
    torch.testing.assert_close(nu2, nu, rtol=rtol, atol=0)
    # the rank-one rows 0..6 are factorised at the rounding noise of their
    # jitter: compare the well-conditioned rows tightly
    torch.testing.assert_close(ld2[7:], logdet[7:], rtol=rtol, atol=rtol * 10)
    torch.testing.assert_close(mm2[7:], mm_ref[7:], rtol=10 * rtol, atol=rtol)
    torch.testing.assert_close(bt[7:], b_ref[7:], rtol=10 * rtol, atol=rtol)
    fin = torch.isfinite(lr_ref)
    assert torch.equal(fin, torch.isfinite(lr2))
    well = fin.clone()
    well[: int(rowptr[7])] = False
    scale = lr_ref[well].abs().max()
    torch.testing.assert_close(lr2[well], lr_ref[well], rtol=10 * rtol, atol=10 * rtol * scale)


# ------------------------------------------- tensor-core (tcgen05) kernels
def tc_problem(D, N=300, k=40, seed=0):
    rng = np.random.default_rng(seed + D)
    X = (rng.standard_normal((N, D)) * 2 + 5).astype(np.float32)  # off-centre: cancellation matters
    graph = O.knn_graph(X, k)
    ((rows, cols),) = O.knn_pattern(graph)
    rowptr = O.ind2ptr(rows, N)
    return rng, X, rowptr, cols


def quad_forms(lr, rowptr, nu, logdet, D):
    """Q = (cst - log rho) / (nu / 2) per pair, in float64."""
    rows = O._rows_of(rowptr)
    cst = O.log_rho_const(nu.astype(np.float64), logdet.astype(np.float64), D)[rows]
    return (cst - lr.astype(np.float64)) / (0.5 * nu[rows].astype(np.float64))


@pytest.mark.parametrize("D", [3, 5, 8, 21, 43, 63, 64])
def test_estep_tc_matches_fp64(K, D):
    rng, X, rowptr, cols = tc_problem(D)
    N = len(X)
    W = (rand_upper(rng, N, D, np.float64) / np.sqrt(D)).astype(np.float32)
    nu = rng.uniform(D + 1, D + 10, N).astype(np.float32)
    logdet = O.chol_logdet(W).astype(np.float32)
    err = torch.zeros(1, dtype=torch.int32, device=DEV)
    order = torch.argsort(torch.tensor(np.diff(rowptr), device=DEV), descending=True).to(torch.int32)
    queue = torch.zeros(1, dtype=torch.int32, device=DEV)
    Wc = K.pack_w_cores(t(W))
    lr = K.estep_tc(t(rowptr), t(cols, torch.int32), t(X), Wc, t(nu), t(logdet), err, order=order, queue=queue)
    assert int(err) == 0
    ref = O.sparse_log_rho(rowptr, cols, X.astype(np.float64), W.astype(np.float64), nu.astype(np.float64),
                           logdet.astype(np.float64))
    lr = lr.cpu().numpy()
    assert np.array_equal(np.isfinite(lr), np.isfinite(ref))
    fin = np.isfinite(ref)
    Q = quad_forms(lr, rowptr, nu, logdet, D)[fin]
    Qr = quad_forms(ref, rowptr, nu, logdet, D)[fin]
    # tf32 hi / lo products: close to fp32 arithmetic (the constant's fp32 rounding included)
    np.testing.assert_allclose(Q, Qr, rtol=2e-5, atol=2e-6 * np.abs(Qr).max())
    # the static schedule (no queue) and an order-less launch give the same values
    lr2 = K.estep_tc(t(rowptr), t(cols, torch.int32), t(X), Wc, t(nu), t(logdet), err)
    np.testing.assert_array_equal(lr2.cpu().numpy(), lr)


@pytest.mark.parametrize("D", [21, 43, 63])
def test_estep_tc_near_singular_whitening(K, D):
    """The precision case of near-singular local covariances: W_triu whitens
    directions of scale 1e-3 (entries near 1e3) and the points sit far from
    the origin, so each product carries ~20 significant bits of cancellation.
    The tf32 hi / lo quad forms stay within a few fp32 roundings of FP64."""
    rng = np.random.default_rng(100 + D)
    N, k, r = 200, 32, max(2, D // 4)
    basis = np.linalg.qr(rng.standard_normal((D, D)))[0]
    z = rng.standard_normal((N, D)) * np.r_[np.ones(r), 1e-3 * np.ones(D - r)]
    X = (z @ basis.T + 20.0).astype(np.float32)
    graph = O.knn_graph(X, k)
    ((rows, cols),) = O.knn_pattern(graph)
    rowptr = O.ind2ptr(rows, N)
    # W_triu of the local covariance basis diag(1, 1e-6) basis^T: L^-T with L = chol
    cov = basis @ np.diag(np.r_[np.ones(r), 1e-6 * np.ones(D - r)]) @ basis.T
    W1 = np.linalg.inv(np.linalg.cholesky(cov)).T
    W = np.repeat(W1[None], N, 0).astype(np.float32)
    nu = np.full(N, D + 2.0, np.float32)
    logdet = O.chol_logdet(W).astype(np.float32)
    err = torch.zeros(1, dtype=torch.int32, device=DEV)
    lr = K.estep_tc(t(rowptr), t(cols, torch.int32), t(X), K.pack_w_cores(t(W)), t(nu), t(logdet), err).cpu().numpy()
    ref = O.sparse_log_rho(rowptr, cols, X.astype(np.float64), W.astype(np.float64), nu.astype(np.float64),
                           logdet.astype(np.float64))
    plain = K.estep_logrho(t(rowptr), t(cols, torch.int32), t(X), t(W), t(nu), t(logdet)).cpu().numpy()
    assert int(err) == 0
    fin = np.isfinite(ref)
    Q = quad_forms(lr, rowptr, nu, logdet, D)[fin]
    Qp = quad_forms(plain, rowptr, nu, logdet, D)[fin]
    Qr = quad_forms(ref, rowptr, nu, logdet, D)[fin]
    err_tc = np.abs(Q - Qr) / np.maximum(Qr, 1.0)
    err_fp32 = np.abs(Qp - Qr) / np.maximum(Qr, 1.0)
    # no worse than a small multiple of the plain FP32 kernel's own error
    assert err_tc.max() <= max(8 * err_fp32.max(), 1e-4), (err_tc.max(), err_fp32.max())


@pytest.mark.parametrize("D", [5, 21, 43, 63, 64])
def test_mstep_tc_matches_fp64(K, D):
    rng, X, rowptr, cols = tc_problem(D, seed=3)
    N = len(X)
    r = rng.uniform(0, 1, size=len(cols)).astype(np.float32)
    err = torch.zeros(1, dtype=torch.int32, device=DEV)
    S, nu = K.mstep_tc(t(rowptr), t(cols, torch.int32), t(r), t(X), D + 1.0, err)
    assert int(err) == 0
    Sr = O.calc_W_inv(rowptr, cols, r.astype(np.float64), X.astype(np.float64), X.astype(np.float64))
    S = S.cpu().numpy()
    scale = np.abs(Sr).max(axis=(1, 2))[:, None, None] + 1e-30
    assert (np.abs(S - Sr) <= 2e-5 * scale).all()
    nur = D + 1.0 + np.bincount(O._rows_of(rowptr), weights=r.astype(np.float64), minlength=N)
    np.testing.assert_allclose(nu.cpu().numpy(), nur, rtol=1e-5)
    # lower_only: the same lower triangle, the upper part left as it was
    S2 = torch.full((N, D, D), 7.0, device=DEV)
    queue = torch.zeros(1, dtype=torch.int32, device=DEV)
    K.mstep_tc(t(rowptr), t(cols, torch.int32), t(r), t(X), D + 1.0, err, S=S2, lower_only=True, queue=queue)
    S2 = S2.cpu().numpy()
    low = np.tril(np.ones((D, D), dtype=bool))
    np.testing.assert_array_equal(S2[:, low], S[:, low])
    assert (S2[:, ~low] == 7.0).all()


def test_mstep_tc_long_rows_accumulate_over_tiles(K):
    """A kernel with more than one 128-pair tile accumulates in tensor memory;
    a row without pairs gets S = 0 and nu = nu_0."""
    rng = np.random.default_rng(4)
    D, N = 30, 5
    X = rng.standard_normal((1000, D)).astype(np.float32)
    counts = np.array([300, 0, 129, 1, 128])
    rowptr = np.concatenate([[0], np.cumsum(counts)])
    cols = rng.integers(0, 1000, size=rowptr[-1])
    r = rng.uniform(0, 1, size=rowptr[-1]).astype(np.float32)
    err = torch.zeros(1, dtype=torch.int32, device=DEV)
    S, nu = K.mstep_tc(t(rowptr), t(cols, torch.int32), t(r), t(X), D + 1.0, err)
    Sr = O.calc_W_inv(rowptr, cols, r.astype(np.float64), X[:N].astype(np.float64), X.astype(np.float64))
    S = S.cpu().numpy()
    for n in range(N):
        sc = np.abs(Sr[n]).max() + 1e-30
        assert np.abs(S[n] - Sr[n]).max() <= 2e-5 * sc
    assert (S[1] == 0).all() and float(nu[1]) == D + 1.0
    assert int(err) == 0


@pytest.mark.parametrize("D,Nq", [(5, 100), (21, 300), (43, 5000), (63, 130), (64, 4097)])
def test_log_pred_density_tc_matches_fp64(K, D, Nq):
    """Tensor-core predictive density: query blocks of 2048 and ragged tiles,
    an odd kernel count, against the float64 restatement and the plain FP32
    kernel."""
    rng = np.random.default_rng(D + Nq)
    N = 777
    X = (rng.standard_normal((N, D)) * 2 + 5).astype(np.float32)
    Y = (X[rng.integers(0, N, Nq)] + 0.3 * rng.standard_normal((Nq, D))).astype(np.float32)
    W = (rand_upper(rng, N, D, np.float64) / np.sqrt(D)).astype(np.float32)
    nu = rng.uniform(D + 1, D + 30, N).astype(np.float32)
    logdet = O.chol_logdet(W).astype(np.float32)
    err = torch.zeros(1, dtype=torch.int32, device=DEV)
    lc = K.pred_coeff(t(nu), t(logdet), D)
    out = K.log_pred_density_tc(t(X), K.pack_w_cores(t(W)), t(nu), lc, t(Y), err)
    assert int(err) == 0
    ref = O.log_pred_density_from_factors(X.astype(np.float64), Y.astype(np.float64), W.astype(np.float64),
                                          nu.astype(np.float64), logdet.astype(np.float64))
    np.testing.assert_allclose(out.cpu().numpy(), ref, rtol=0, atol=1e-3)
    plain = K.log_pred_density(t(X), t(W), t(nu), lc, t(Y))
    assert float((out - plain).abs().max()) <= 1e-3


# ------------------------------------------------------------ tiled layout
def tf32_rna(x):
    """Round float32 to the nearest tf32 (ties away from zero) by bit arithmetic."""
    return ((x.view(torch.int32) + 0x1000) & ~0x1FFF).view(torch.float32)


def w_cores_ref(W, D):
    """The W-cores layout of W_triu [N, D, D] (float32, on the device) built with
    torch: X = W_triu^T, per column block J the tf32 hi parts of row blocks
    I >= J, then their lo parts (tf32 of X - hi), each block as the two
    K-major 8 x 4 cores of its columns 8J..8J+3 and 8J+4..8J+7."""
    N = W.shape[0]
    nt = 1 if D <= 8 else {16: 2, 24: 3, 32: 4, 48: 6, 64: 8}[next(p for p in (16, 24, 32, 48, 64) if D <= p)]
    Xp = torch.zeros(N, 8 * nt, 8 * nt, device=W.device)
    Xp[:, :D, :D] = torch.tril(W.mT)
    hi = tf32_rna(Xp)
    lo = tf32_rna(Xp - hi)
    segs = []
    for J in range(nt):
        for part in (hi, lo):
            for I in range(J, nt):
                for h in range(2):
                    segs.append(part[:, 8 * I:8 * I + 8, 8 * J + 4 * h:8 * J + 4 * h + 4].reshape(N, 32))
    return torch.cat(segs, dim=1).contiguous()


@pytest.mark.parametrize("D", [3, 8, 13, 21, 36, 43, 63, 64])
def test_pack_w_cores_layout(K, D):
    rng = np.random.default_rng(D)
    W = t((rand_upper(rng, 20, D, np.float64)).astype(np.float32))
    Wc = K.pack_w_cores(W)
    torch.testing.assert_close(Wc, w_cores_ref(W, D), rtol=0, atol=0)


def spd_lowrank(rng, N, D, rank):
    A = rng.standard_normal((N, D, rank))
    return A @ np.swapaxes(A, 1, 2) / rank


@pytest.mark.parametrize("D", [13, 21, 43, 63, 64])
def test_factor_tiled_equals_dense_layout(K, D):
    """Bulk-copied tiles (S and P interleaved, T as tiles) give the dense
    layout's factorisation bit for bit, jitter ladder included, and both
    write the same W cores."""
    rng = np.random.default_rng(D)
    N = 150
    S = spd_lowrank(rng, N, D, D).astype(np.float32)
    S[:20] = spd_lowrank(rng, 20, D, 3).astype(np.float32)  # rank-deficient: the prior carries them
    S[20:25] = spd_lowrank(rng, 5, D, 2).astype(np.float32)
    P = spd_lowrank(rng, N, D, D + 2).astype(np.float32)
    P[20:25] = spd_lowrank(rng, 5, D, 2).astype(np.float32)  # A singular without jitter: the ladder runs
    Tm = np.linalg.cholesky(P.astype(np.float64) + 1e-3 * np.eye(D)).astype(np.float32)
    a = rng.uniform(1, 3, N).astype(np.float32)
    b = rng.uniform(1, 3, N).astype(np.float32)
    nu0 = torch.tensor([D + 1.5], device=DEV)
    jit1 = t(np.zeros(N, np.float32))
    Wc1 = K.w_cores_like(D, N, DEV)
    W1, ld1, info1, _, tr1 = K.posterior_factor(t(S), jit1, 1.2e-7, P=t(P), nu_0=nu0, a=t(a), b=t(b), T=t(Tm),
                                                T_lower=True, W_cores=Wc1)
    nt = K.tile_count(D)
    SP = torch.zeros(N, nt * 128, device=DEV)
    Tt = torch.zeros(N, nt * 64, device=DEV)
    K.pack_tiles(t(S), SP, 128, 0)
    K.pack_tiles(t(P), SP, 128, 64)
    K.pack_tiles(t(Tm), Tt, 64, 0)
    jit2 = t(np.zeros(N, np.float32))
    W2, ld2, tr2 = torch.empty_like(W1), torch.empty_like(ld1), torch.empty_like(tr1)
    info2 = torch.empty_like(info1)
    Xt = torch.full((N, nt * 64), 5.0, device=DEV)
    Wc = torch.full_like(Wc1, 5.0)
    K.posterior_factor_tiled(SP, D, jit2, 1.2e-7, nu0, t(a), t(b), W2, ld2, info2, T_tiles=Tt, trace=tr2,
                             X_tiles=Xt, W_cores=Wc)
    # X = W_triu^T as lower tiles
    ref = torch.zeros(N, nt * 64, device=DEV)
    K.pack_tiles(W1.mT.contiguous(), ref, 64, 0)
    torch.testing.assert_close(Xt, ref, rtol=0, atol=0)
    # the W cores of W_triu, from the tiled and the dense factorisation
    torch.testing.assert_close(Wc, w_cores_ref(W1, D), rtol=0, atol=0, equal_nan=True)
    torch.testing.assert_close(Wc1, Wc, rtol=0, atol=0, equal_nan=True)
    # the cores alone (no dense or tiled float output)
    Wc2 = torch.zeros_like(Wc)
    jit3 = t(np.zeros(N, np.float32))
    K.posterior_factor_tiled(SP, D, jit3, 1.2e-7, nu0, t(a), t(b), None, torch.empty_like(ld1),
                             torch.empty_like(info1), W_cores=Wc2)
    torch.testing.assert_close(Wc2, Wc, rtol=0, atol=0, equal_nan=True)
    assert (jit1[20:25] > 0).all()
    torch.testing.assert_close(info2, info1, rtol=0, atol=0)
    torch.testing.assert_close(jit2, jit1, rtol=0, atol=0)
    torch.testing.assert_close(W2, W1, rtol=0, atol=0, equal_nan=True)
    torch.testing.assert_close(ld2, ld1, rtol=0, atol=0, equal_nan=True)
    torch.testing.assert_close(tr2, tr1, rtol=0, atol=0, equal_nan=True)


@pytest.mark.parametrize("D", [13, 21, 36, 43, 63, 64])
def test_mstep_tc_tiled_equals_rows(K, D):
    """The tiled M-step equals the dense one bit for bit (every tile written,
    zero outside D and above the diagonal)."""
    rng, X, rowptr, cols = tc_problem(D, seed=5)
    N = len(X)
    r = rng.uniform(0, 1, size=len(cols)).astype(np.float32)
    err = torch.zeros(1, dtype=torch.int32, device=DEV)
    S, nu = K.mstep_tc(t(rowptr), t(cols, torch.int32), t(r), t(X), D + 1.0, err)
    nt = K.tile_count(D)
    ref = torch.zeros(N, nt * 128, device=DEV)
    K.pack_tiles(S, ref, 128, 0)
    SP = torch.full((N, nt * 128), 3.0, device=DEV)
    nu2 = torch.empty_like(nu)
    K.mstep_tc_tiled(t(rowptr), t(cols, torch.int32), t(r), t(X), D + 1.0, err, SP, nu2)
    assert int(err) == 0
    view = SP.view(N, nt, 2, 64)
    torch.testing.assert_close(view[:, :, 0], ref.view(N, nt, 2, 64)[:, :, 0], rtol=0, atol=0)
    assert (view[:, :, 1] == 3.0).all()  # the P halves are left alone
    torch.testing.assert_close(nu2, nu, rtol=0, atol=0)


@pytest.mark.parametrize("D", [13, 21, 36, 43, 63, 64])
def test_estep_tc_kernel_offset(K, D):
    """The E-step over rows 7.. of the CSR as a second launch (kernel_offset 7,
    its own cores) gives the same values as the whole launch."""
    rng, X, rowptr, cols = tc_problem(D, seed=9)
    N = len(X)
    W = (rand_upper(rng, N, D, np.float64) / np.sqrt(D)).astype(np.float32)
    nu = rng.uniform(D + 1, D + 10, N).astype(np.float32)
    logdet = O.chol_logdet(W).astype(np.float32)
    err = torch.zeros(1, dtype=torch.int32, device=DEV)
    Wc = K.pack_w_cores(t(W))
    lr = K.estep_tc(t(rowptr), t(cols, torch.int32), t(X), Wc, t(nu), t(logdet), err)
    lr3 = K.estep_tc(t(rowptr[7:] - rowptr[7]), t(cols[rowptr[7]:], torch.int32), t(X), Wc[7:].contiguous(),
                     t(nu[7:]), t(logdet[7:]), err, kernel_offset=7)
    assert int(err) == 0
    torch.testing.assert_close(lr3, lr[rowptr[7]:], rtol=0, atol=0)
    # rows of X already 16-byte aligned (a padded buffer's view) give the same values
    Xp = K.pad_rows(t(X))
    lr4 = K.estep_tc(t(rowptr), t(cols, torch.int32), Xp, Wc, t(nu), t(logdet), err)
    torch.testing.assert_close(lr4, lr, rtol=0, atol=0)


def test_bounded_wait_times_out_sets_err_and_the_engine_raises(K):
    """A tensor-core completion wait that runs out: the test hook makes the
    first stage's mbarrier expect 16 bytes no copy delivers (every issued copy
    lands, nothing stays in flight).  The kernel gives up after its time
    limit, sets err, frees its tensor memory and returns; the engine's error
    check then raises, and the context stays usable."""
    from lakde_b200 import _native as nat
    from lakde_b200.engine import FusedKNN
    from lakde_b200.sparse_util import PairPattern

    rng, X, rowptr, cols = tc_problem(21, N=64, k=8)
    N, D = X.shape
    W = (rand_upper(rng, N, D, np.float64) / np.sqrt(D)).astype(np.float32)
    nu = t(rng.uniform(D + 1, D + 10, N).astype(np.float32))
    logdet = t(O.chol_logdet(W).astype(np.float32))
    Xp = K.pad_rows(t(X))
    Wc = K.pack_w_cores(t(W))
    out = torch.zeros(len(cols), device=DEV)
    Xt = t(X)
    graph = torch.tensor(O.knn_graph(X, 8).astype(np.int32), device=DEV)
    tiny = torch.tensor(1e-6, device=DEV)
    eng = FusedKNN(Xt, graph, PairPattern.from_knn_graph(graph), float(D), tiny, tiny, 0.0, 8)
    eng.check_errors()
    # the device buffers stay referenced until the launch has completed
    rowptr_d, cols_d = t(rowptr), t(cols, torch.int32)
    st = nat.lib().lakde_tc_wait_timeout_probe(N, D, N, nat.ptr(rowptr_d), nat.ptr(cols_d), nat.ptr(Xp),
                                               Xp.stride(0), nat.ptr(Wc), nat.ptr(nu), nat.ptr(logdet),
                                               nat.ptr(out), nat.ptr(eng.err), nat.stream_of(out))
    nat.check(st, "tc_wait_timeout_probe")
    torch.cuda.synchronize()
    assert int(eng.err) == 1
    with pytest.raises(RuntimeError, match="timed out"):
        eng.check_errors()
    # the device still works: an ordinary launch afterwards gives correct values
    err = torch.zeros(1, dtype=torch.int32, device=DEV)
    lr = K.estep_tc(t(rowptr), t(cols, torch.int32), Xt, Wc, nu, logdet, err)
    ref = O.sparse_log_rho(rowptr, cols, X.astype(np.float64), W.astype(np.float64),
                           nu.cpu().numpy().astype(np.float64), logdet.cpu().numpy().astype(np.float64))
    assert int(err) == 0
    fin = np.isfinite(ref)
    np.testing.assert_allclose(lr.cpu().numpy()[fin], ref[fin], rtol=1e-4, atol=1e-3)


@pytest.mark.parametrize("D,N,dtype", [(3, 500, np.float64), (21, 3000, np.float32), (43, 1000, np.float32),
                                       (64, 777, np.float64), (43, 0, np.float32)])
def test_weighted_gram_matches_fp64(K, D, N, dtype):
    """sum_n w_n W_triu_n W_triu_n^T of the hierarchical shared precision
    (lakde/local_hierarchical_kde.py:293-297) against a float64 einsum."""
    rng = np.random.default_rng(D + N)
    W = np.triu(rng.standard_normal((N, D, D))).astype(dtype)
    w = rng.uniform(0.5, 30, N).astype(dtype)
    out = K.weighted_gram(t(W), t(w)).cpu().numpy()
    ref = np.einsum("n,nij,nkj->ik", w.astype(np.float64), W.astype(np.float64), W.astype(np.float64))
    np.testing.assert_allclose(out, ref, rtol=1e-12, atol=1e-10 * max(1.0, np.abs(ref).max()))
    np.testing.assert_array_equal(out, out.T)
