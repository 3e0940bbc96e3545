"""Generate the golden vectors that pin the oracle to the reference.

Runs the reference implementation itself (falkaer/lakde, torch CPU path with
LAKDE_NO_EXT=1) on small seeded inputs and stores inputs and outputs as
.npz files next to this script.  Only this script reads the reference
checkout; the tests read the .npz files.

    python tests/golden/make_golden.py path/to/lakde-checkout
    LAKDE_REFERENCE=path/to/lakde-checkout python tests/golden/make_golden.py

GOLDEN_ONLY=ops|models|checkpoint regenerates one group of fixtures.
"""

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("LAKDE_REFERENCE")
if not REF or not os.path.isdir(os.path.join(REF, "lakde")):
    sys.exit("usage: make_golden.py path/to/lakde-checkout (or set LAKDE_REFERENCE)")
os.environ["LAKDE_NO_EXT"] = "1"
sys.path.insert(0, REF)
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import torch  # noqa: E402

from lakde import LocalHierarchicalKDE, LocalKNearestKDE  # noqa: E402
from lakde import kernels as ref_kernels  # noqa: E402
from lakde import linalg_util as ref_linalg  # noqa: E402
from lakde import sparse_util as ref_sparse  # noqa: E402
from lakde import utils as ref_utils  # noqa: E402

from lakde_b200.synthetic import circle_gmm  # noqa: E402

torch.set_num_threads(8)


def t2n(t):
    return t.detach().cpu().numpy()


def ops_fixtures():
    rng = np.random.default_rng(1234)
    out = {}
    for dt_name, dt in (("f32", torch.float32), ("f64", torch.float64)):
        for D in (1, 2, 5, 8, 17, 33):
            N, M = 7, 11
            W = np.triu(rng.standard_normal((N, D, D)))
            W[:, np.arange(D), np.arange(D)] = np.abs(W[:, np.arange(D), np.arange(D)]) + 0.5
            Xn = rng.standard_normal((N, D))
            Xm = rng.standard_normal((M, D))
            Wt, Xnt, Xmt = (torch.tensor(a, dtype=dt) for a in (W, Xn, Xm))
            Q = ref_kernels.chol_quad_form(Wt, Xnt, Xmt)
            key = f"quad_{dt_name}_d{D}"
            out[key + "_W"] = t2n(Wt)
            out[key + "_Xn"] = t2n(Xnt)
            out[key + "_Xm"] = t2n(Xmt)
            out[key + "_Q"] = t2n(Q)
        for D in (1, 3, 7, 16):
            N, M = 9, 40
            counts = rng.integers(0, 12, size=N)
            counts[2] = 0
            counts[-1] = 0
            row = np.repeat(np.arange(N), counts)
            col = rng.integers(0, M, size=len(row))
            val = rng.uniform(0, 1, size=len(row))
            rowptr = np.concatenate([[0], np.cumsum(counts)])
            Xn = rng.standard_normal((N, D))
            Xm = rng.standard_normal((M, D))
            args = (
                torch.tensor(rowptr, dtype=torch.int64),
                torch.tensor(col, dtype=torch.int64),
                torch.tensor(val, dtype=dt),
                torch.tensor(Xn, dtype=dt),
                torch.tensor(Xm, dtype=dt),
            )
            S = ref_kernels.calc_W_inv(*args)
            key = f"winv_{dt_name}_d{D}"
            for name, a in zip(("rowptr", "col", "value", "Xn", "Xm"), args):
                out[f"{key}_{name}"] = t2n(a)
            out[key + "_S"] = t2n(S)
        # jittered Cholesky: PD, rank-deficient and indefinite matrices
        D = 6
        mats = []
        for i in range(8):
            A = rng.standard_normal((D, D if i < 4 else 3))
            S = A @ A.T
            if i == 6:
                S -= 1e-12 * np.eye(D)
            if i == 7:
                S *= 1e3
            mats.append(S)
        X = torch.tensor(np.stack(mats), dtype=dt)
        L, jit = ref_linalg.stabilized_cholesky(X, X.new_zeros(8))
        out[f"chol_{dt_name}_X"] = t2n(X)
        out[f"chol_{dt_name}_L"] = t2n(L)
        out[f"chol_{dt_name}_jitter"] = t2n(jit)
        a = torch.tensor(rng.uniform(2.5, 40, size=13), dtype=dt)
        for D in (1, 2, 8, 21):
            out[f"special_{dt_name}_a"] = t2n(a)
            out[f"special_{dt_name}_mvdigamma_d{D}"] = t2n(ref_linalg.mvdigamma(a, D))
            out[f"special_{dt_name}_mvlgamma_d{D}"] = t2n(ref_linalg.mvlgamma(a, D))
    # ind2ptr
    row = np.sort(rng.integers(0, 50, size=300))
    row = row[(row != 7) & (row != 8)]
    out["ind2ptr_row"] = row.astype(np.int32)
    out["ind2ptr_M"] = np.array(60)
    out["ind2ptr_out"] = t2n(ref_kernels.ind2ptr(torch.tensor(row, dtype=torch.int64), 60))
    # kNN graph and COO pattern
    Xk = rng.standard_normal((300, 3)).astype(np.float32)
    for inc in (False, True):
        g = ref_utils.compute_knn_graph(torch.tensor(Xk), 10, 64, include_self=inc, dtype=torch.int32)
        out[f"knn_self{int(inc)}"] = t2n(g)
        slices = ref_sparse.graph_to_slices(g, 128)
        for bi, s in enumerate(slices):
            out[f"pattern_self{int(inc)}_b{bi}"] = t2n(s)
    out["knn_X"] = Xk
    np.savez_compressed(os.path.join(HERE, "ops.npz"), **out)


class Recorder:
    def __init__(self):
        self.elbo = []

    def __call__(self, X, model, it):
        self.elbo.append(float(model.compute_elbo(X)))


def run_model(cls, X, Y, dtype, iterations, threshold, block_size, **kw):
    Xt = torch.tensor(X, dtype=dtype)
    Yt = torch.tensor(Y, dtype=dtype)
    m = cls(block_size=block_size, **kw)
    rec = Recorder()
    m.fit(Xt, iterations=iterations, callbacks=rec, sparsity_threshold=threshold)
    ll = m.log_pred_density(Xt, Yt)
    res = {
        "X": X,
        "Y": Y,
        "elbo": np.array(rec.elbo),
        "c": t2n(m.rnm_log_consts),
        "nu": t2n(m.nu),
        "logdet_W": t2n(m.logdet_W),
        "b": t2n(m.b),
        "W_inv_jitter": t2n(m.W_inv_jitter),
        "ll": t2n(ll),
        "nnz": np.array(sum(v.numel() for _, v in m.rnm_blocks)),
    }
    return m, res


def model_fixtures():
    Xtr, Xte = circle_gmm(seed=0, n_train=2000, n_test=1000)
    for name, dt, B, thr in (
        ("knn_c1_f32_bN", torch.float32, 2000, None),
        ("knn_c1_f32_b512", torch.float32, 512, None),
        ("knn_c1_f32_bN_t5e-4", torch.float32, 2000, 5e-4),
        ("knn_c1_f64_bN", torch.float64, 2000, None),
    ):
        m, res = run_model(LocalKNearestKDE, Xtr, Xte, dt, 10, thr, B, k_or_knn_graph=20)
        res["knn_graph"] = t2n(m.knn_graph)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **res)
        print(name, res["elbo"][-1], res["ll"].mean(), int(res["nnz"]))
    # a small case keeping the full responsibility state
    Xs, Ys = circle_gmm(seed=3, n_train=400, n_test=100)
    for name, dt, B in (("knn_small_f32_bN", torch.float32, 400), ("knn_small_f32_b128", torch.float32, 128),
                        ("knn_small_f64_bN", torch.float64, 400)):
        m, res = run_model(LocalKNearestKDE, Xs, Ys, dt, 4, 1e-4, B, k_or_knn_graph=10)
        rows, cols, vals = [], [], []
        for bi, (ind, v) in enumerate(m.rnm_blocks):
            rows.append(t2n(ind[0]).astype(np.int64) + bi * m.block_size)
            cols.append(t2n(ind[1]))
            vals.append(t2n(v))
        res["r_row"] = np.concatenate(rows)
        res["r_col"] = np.concatenate(cols)
        res["r_val"] = np.concatenate(vals)
        res["knn_graph"] = t2n(m.knn_graph)
        res["sigma_0_jitter"] = t2n(m.sigma_0_jitter)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **res)
        print(name, res["elbo"][-1], res["ll"].mean(), int(res["nnz"]))
    # hierarchical model, 3-d
    rng = np.random.default_rng(5)
    means = rng.standard_normal((4, 3)) * 2
    lab = rng.integers(0, 4, size=700)
    Z = means[lab] + rng.standard_normal((700, 3)) @ np.diag([0.3, 0.2, 0.05])
    Xh, Yh = Z[:500].astype(np.float32), Z[500:].astype(np.float32)
    for name, dt, B in (("hier_f32_bN", torch.float32, 500), ("hier_f32_b128", torch.float32, 128),
                        ("hier_f64_bN", torch.float64, 500)):
        m, res = run_model(LocalHierarchicalKDE, Xh, Yh, dt, 5, None, B, k_or_knn_graph=15)
        res["W_shared_triu"] = t2n(m.W_shared_triu)
        res["expect_lambda_contribs"] = t2n(m.expect_lambda_contribs)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **res)
        print(name, res["elbo"][-1], res["ll"].mean(), int(res["nnz"]))


def state_to_arrays(state, prefix="state_"):
    """A reference state dict as flat npz arrays (rnm_blocks block by block),
    copied: the reference's state dict holds its live tensors, which a
    continued fit updates in place."""
    out = {}
    for key, v in state.items():
        if key == "rnm_blocks":
            out[prefix + "rnm_nblocks"] = np.array(len(v))
            for bi, (ind, val) in enumerate(v):
                out[f"{prefix}rnm_b{bi}_ind"] = t2n(ind).copy()
                out[f"{prefix}rnm_b{bi}_val"] = t2n(val).copy()
        elif torch.is_tensor(v):
            out[prefix + key] = t2n(v).copy()
        else:
            out[prefix + key] = np.array(v)
    return out


def checkpoint_fixtures():
    """The reference's state dict after 5 iterations of the config-1 run
    (block_size 512, float32), then the ELBO after every block update and the
    held-out log density of 5 more iterations of the same model object."""
    Xtr, Xte = circle_gmm(seed=0, n_train=2000, n_test=1000)
    Xt, Yt = torch.tensor(Xtr), torch.tensor(Xte)
    m = LocalKNearestKDE(block_size=512, k_or_knn_graph=20)
    m.fit(Xt, iterations=5, sparsity_threshold=None)
    res = state_to_arrays(m.state_dict())
    res["elbo_at_state"] = np.array(float(m.compute_elbo(Xt)))
    rec = Recorder()
    m.fit(Xt, iterations=5, callbacks=rec, sparsity_threshold=None)
    res.update(X=Xtr, Y=Xte, elbo_after=np.array(rec.elbo), ll_after=t2n(m.log_pred_density(Xt, Yt)),
               c_after=t2n(m.rnm_log_consts))
    np.savez_compressed(os.path.join(HERE, "knn_c1_f32_b512_resume.npz"), **res)
    print("knn_c1_f32_b512_resume", res["elbo_after"][-1], res["ll_after"].mean())


if __name__ == "__main__":
    only = os.environ.get("GOLDEN_ONLY")
    if only in (None, "ops"):
        ops_fixtures()
    if only in (None, "models"):
        model_fixtures()
    if only in (None, "checkpoint"):
        checkpoint_fixtures()
