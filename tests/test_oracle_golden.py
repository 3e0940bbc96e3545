"""Pins the CPU oracle to the reference: every oracle function is checked
against golden vectors produced by running the reference implementation
itself (tests/golden/make_golden.py)."""

import os

import numpy as np
import pytest

from oracle import lakde_oracle as O

from .conftest import GOLDEN


def load(name):
    return np.load(os.path.join(GOLDEN, name + ".npz"))


@pytest.fixture(scope="module")
def ops():
    return load("ops")


@pytest.mark.parametrize("dt", ["f32", "f64"])
@pytest.mark.parametrize("D", [1, 2, 5, 8, 17, 33])
def test_quad_form(ops, dt, D):
    k = f"quad_{dt}_d{D}"
    Q = O.chol_quad_form(ops[k + "_W"], ops[k + "_Xn"], ops[k + "_Xm"])
    rtol = 1e-5 if dt == "f32" else 1e-12
    np.testing.assert_allclose(Q, ops[k + "_Q"], rtol=rtol, atol=rtol)


@pytest.mark.parametrize("dt", ["f32", "f64"])
@pytest.mark.parametrize("D", [1, 3, 7, 16])
def test_scatter_cov(ops, dt, D):
    k = f"winv_{dt}_d{D}"
    S = O.calc_W_inv(*(ops[f"{k}_{n}"] for n in ("rowptr", "col", "value", "Xn", "Xm")))
    rtol = 1e-5 if dt == "f32" else 1e-12
    np.testing.assert_allclose(S, ops[k + "_S"], rtol=rtol, atol=rtol)


def test_ind2ptr(ops):
    out = O.ind2ptr(ops["ind2ptr_row"], int(ops["ind2ptr_M"]))
    np.testing.assert_array_equal(out, ops["ind2ptr_out"])
    np.testing.assert_array_equal(O.ind2ptr(np.zeros(0, np.int64), 5), np.zeros(6))


@pytest.mark.parametrize("dt", ["f32", "f64"])
def test_jittered_cholesky(ops, dt):
    X = ops[f"chol_{dt}_X"]
    L, jit = O.stabilized_cholesky(X, np.zeros(len(X), X.dtype))
    ref = ops[f"chol_{dt}_jitter"]
    # ladder values are eps * (2^(k+1) - 1); rank-deficient matrices sit at the
    # rounding noise of the factorisation, so their rung may differ by up to
    # two doublings from LAPACK's
    eps = np.finfo(X.dtype).eps
    k = np.log2(jit / eps + 1)
    nz = jit != 0
    np.testing.assert_allclose(k[nz], np.round(k[nz]), atol=1e-9)
    np.testing.assert_array_equal(jit == 0, ref == 0)
    kr = np.log2(ref[nz] / eps + 1)
    assert np.abs(k[nz] - kr).max() <= 2
    # the matrix shifted by -1e-12 I (well above the rounding noise in float64)
    # lands on the same rung
    if dt == "f64":
        assert jit[6] == ref[6]
    same = jit == ref
    rtol = 2e-3 if dt == "f32" else 1e-8
    np.testing.assert_allclose(L[same], ops[f"chol_{dt}_L"][same], rtol=rtol, atol=rtol * np.abs(L).max())


@pytest.mark.parametrize("dt", ["f32", "f64"])
@pytest.mark.parametrize("D", [1, 2, 8, 21])
def test_special_functions(ops, dt, D):
    a = ops[f"special_{dt}_a"]
    rtol = 2e-6 if dt == "f32" else 1e-12
    np.testing.assert_allclose(O.mvdigamma(a, D), ops[f"special_{dt}_mvdigamma_d{D}"], rtol=rtol)
    np.testing.assert_allclose(O.mvlgamma(a, D), ops[f"special_{dt}_mvlgamma_d{D}"], rtol=rtol)


@pytest.mark.parametrize("self_", [0, 1])
def test_knn_graph_and_pattern(ops, self_):
    X = ops["knn_X"]
    ref = ops[f"knn_self{self_}"]
    g = O.knn_graph(X, 10, include_self=bool(self_))
    # the reference ranks fp32 cdist distances; the oracle ranks exact ones.
    # Away from near-ties they agree position by position.
    assert_same_neighbours(X, g, ref, min_agree=0.97)
    pats = O.knn_pattern(ref, 128)
    for bi, p in enumerate(pats):
        r = ops[f"pattern_self{self_}_b{bi}"]
        # same pairs; within a row the reference order is arbitrary
        key = lambda a: np.lexsort((a[1], a[0]))
        np.testing.assert_array_equal(p[:, key(p)], r[:, key(r)])


def _fit(name, cls, iters, thr, B, k, **kw):
    g = load(name)
    dt = g["X"].dtype if "f32" in name else np.float64
    X = g["X"].astype(dt)
    Y = g["Y"].astype(dt)
    m = cls(k=k, block_size=B, **kw)
    el = []
    m.fit(X, iterations=iters, threshold=thr, callback=lambda mm, XX: el.append(mm.compute_elbo(XX)))
    return m, g, np.array(el), m.log_pred_density(X, Y)


CASES = [
    ("knn_small_f32_bN", O.KNNKDEOracle, 4, 1e-4, 400, 10, 1e-6),
    ("knn_small_f32_b128", O.KNNKDEOracle, 4, 1e-4, 128, 10, 1e-6),
    ("knn_small_f64_bN", O.KNNKDEOracle, 4, 1e-4, 400, 10, 1e-12),
    ("hier_f32_bN", O.HierKDEOracle, 5, None, 500, 15, 1e-6),
    ("hier_f32_b128", O.HierKDEOracle, 5, None, 128, 15, 5e-5),
    ("hier_f64_bN", O.HierKDEOracle, 5, None, 500, 15, 1e-12),
]


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_model_trajectory(case):
    name, cls, iters, thr, B, k, rtol = case
    m, g, elbo, ll = _fit(name, cls, iters, thr, B, k)
    np.testing.assert_allclose(elbo, g["elbo"], rtol=rtol)
    atol = 1e3 * rtol
    np.testing.assert_allclose(m.rnm_log_consts, g["c"], atol=atol)
    np.testing.assert_allclose(m.nu, g["nu"], rtol=atol)
    np.testing.assert_allclose(m.logdet_W, g["logdet_W"], atol=atol)
    np.testing.assert_allclose(m.b, g["b"], rtol=atol)
    np.testing.assert_allclose(ll, g["ll"], atol=atol)
    assert sum(v.size for _, v in m.rnm_blocks) == int(g["nnz"])
    if "r_val" in g:
        rows = np.concatenate([ix[0].astype(np.int64) + bi * m.block_size for bi, (ix, _) in enumerate(m.rnm_blocks)])
        cols = np.concatenate([ix[1] for ix, _ in m.rnm_blocks])
        vals = np.concatenate([v for _, v in m.rnm_blocks])
        mine = np.lexsort((cols, rows))
        ref = np.lexsort((g["r_col"], g["r_row"]))
        np.testing.assert_array_equal(rows[mine], g["r_row"][ref])
        np.testing.assert_array_equal(cols[mine], g["r_col"][ref])
        np.testing.assert_allclose(vals[mine], g["r_val"][ref], rtol=atol, atol=atol * 1e-3)


@pytest.mark.parametrize("name,dt", [("knn_c1_f32_bN", np.float32), ("knn_c1_f64_bN", np.float64)])
def test_config1_trajectory(name, dt):
    """d=2, N=2,000, K=20, 10 iterations at block_size = N (the batch schedule)."""
    g = load(name)
    m = O.KNNKDEOracle(k=20, block_size=2000)
    el = []
    X = g["X"].astype(dt)
    m.fit(X, iterations=10, callback=lambda mm, XX: el.append(mm.compute_elbo(XX)))
    rtol = 1e-6 if dt == np.float32 else 1e-12
    np.testing.assert_allclose(el, g["elbo"], rtol=rtol)
    assert_same_neighbours(X, m.knn_graph, g["knn_graph"])


def assert_same_neighbours(X, mine, ref, min_agree=0.99):
    """Graphs agree position by position except between near-tied distances.

    The reference ranks float32 cdist distances computed as |a|^2 + |b|^2 - 2ab,
    whose absolute error in d^2 is about eps32 * (|a|^2 + |b|^2); neighbours
    whose exact squared distances differ by less than that may swap.
    """
    agree = (mine == ref).all(1)
    assert agree.mean() >= min_agree
    X64 = X.astype(np.float64)
    sq = (X64**2).sum(-1)
    eps32 = np.finfo(np.float32).eps
    for r in np.nonzero(~agree)[0]:
        dm = ((X64[mine[r]] - X64[r]) ** 2).sum(-1)
        dr = ((X64[ref[r]] - X64[r]) ** 2).sum(-1)
        tol = 64 * eps32 * (sq[r] + sq.max())
        np.testing.assert_allclose(dm, dr, rtol=0, atol=tol)
