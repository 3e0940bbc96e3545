"""Backward of the predictive log density: the hand-written CUDA pass against
torch autograd through a functional restatement of the reference formula
(lakde/local_adaptive_kde.py:209-223 with the fallback quad form of
lakde/kernels.py:20-23), and against float64 central finite differences
(h = 1e-4, relative error <= 1e-4)."""

import math

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def torch_reference(X, L, nu, Y):
    """The reference formula as a differentiable torch function (float64, CPU)."""
    N, D = X.shape
    W_triu = torch.linalg.inv(L).mT
    logdet = 2 * torch.log(torch.diagonal(W_triu, dim1=-2, dim2=-1)).sum(-1)
    lc = torch.lgamma((nu + 1) / 2) - torch.lgamma((nu + 1 - D) / 2) + 0.5 * logdet - D / 2 * math.log(math.pi)
    diff = Y[None, :, :] - X[:, None, :]
    z = (W_triu.mT @ diff.mT).mT
    Q = (z * z).sum(-1)
    lp = lc[:, None] - (nu[:, None] + 1) / 2 * torch.log1p(Q)
    return -math.log(N) + torch.logsumexp(lp, dim=0)


def problem(D, N=60, Nq=25, seed=0):
    rng = np.random.default_rng(seed + D)
    X = rng.standard_normal((N, D))
    Y = X[rng.integers(0, N, Nq)] + 0.3 * rng.standard_normal((Nq, D))
    A = rng.standard_normal((N, D, D)) * 0.3
    L = np.tril(A)
    L[:, np.arange(D), np.arange(D)] = np.abs(L[:, np.arange(D), np.arange(D)]) + 0.5
    nu = rng.uniform(D + 1, D + 20, N)
    g = rng.standard_normal(Nq)
    return [torch.tensor(a, dtype=torch.float64) for a in (X, L, nu, Y, g)]


@pytest.mark.parametrize("D", [1, 3, 8, 21])
def test_matches_torch_autograd(D):
    from lakde_b200.grad import log_pred_density

    X, L, nu, Y, g = problem(D)
    Yr = Y.clone().requires_grad_(True)
    Lr = L.clone().requires_grad_(True)
    ref = torch_reference(X, Lr, nu, Yr)
    (ref * g).sum().backward()
    Yc = Y.cuda().requires_grad_(True)
    Lc = L.cuda().requires_grad_(True)
    out = log_pred_density(X.cuda(), Lc, nu.cuda(), Yc)
    (out * g.cuda()).sum().backward()
    torch.testing.assert_close(out.cpu(), ref.detach(), rtol=1e-10, atol=1e-10)
    torch.testing.assert_close(Yc.grad.cpu(), Yr.grad, rtol=1e-8, atol=1e-10)
    torch.testing.assert_close(Lc.grad.cpu(), torch.tril(Lr.grad), rtol=1e-8, atol=1e-10)


@pytest.mark.parametrize("D", [3, 8])
def test_central_finite_differences(D):
    from lakde_b200.grad import log_pred_density

    X, L, nu, Y, g = problem(D, seed=5)
    Xc, nuc, gc = X.cuda(), nu.cuda(), g.cuda()
    Yc = Y.cuda().requires_grad_(True)
    Lc = L.cuda().requires_grad_(True)
    (log_pred_density(Xc, Lc, nuc, Yc) * gc).sum().backward()
    f = lambda Lx, Yx: float((log_pred_density(Xc, Lx, nuc, Yx) * gc).sum())  # noqa: E731
    h = 1e-4
    rng = np.random.default_rng(1)
    for _ in range(6):
        q, d = int(rng.integers(len(Y))), int(rng.integers(D))
        e = torch.zeros_like(Yc)
        e[q, d] = h
        fd = (f(Lc.detach(), Yc.detach() + e) - f(Lc.detach(), Yc.detach() - e)) / (2 * h)
        an = float(Yc.grad[q, d])
        assert abs(fd - an) <= 1e-4 * max(abs(an), 1e-3), (fd, an)
        n, i = int(rng.integers(len(X))), int(rng.integers(D))
        j = int(rng.integers(i + 1))
        e = torch.zeros_like(Lc)
        e[n, i, j] = h
        fd = (f(Lc.detach() + e, Yc.detach()) - f(Lc.detach() - e, Yc.detach())) / (2 * h)
        an = float(Lc.grad[n, i, j])
        assert abs(fd - an) <= 1e-4 * max(abs(an), 1e-3), (fd, an)


def test_float32_gradients_close_to_float64():
    from lakde_b200.grad import log_pred_density

    X, L, nu, Y, g = problem(8, N=500, Nq=300)
    grads = []
    for dt in (torch.float64, torch.float32):
        Yc = Y.to("cuda", dt).requires_grad_(True)
        Lc = L.to("cuda", dt).requires_grad_(True)
        (log_pred_density(X.to("cuda", dt), Lc, nu.to("cuda", dt), Yc) * g.to("cuda", dt)).sum().backward()
        grads.append((Yc.grad.double().cpu(), Lc.grad.double().cpu()))
    for a, b in zip(*grads):
        err = (a - b).abs().max() / a.abs().max()
        assert err < 1e-4, float(err)


def test_fitted_d21_model_gradients_match_fp64_finite_differences():
    """The backward workload at d=21: LocalKNearestKDE fitted (K=64, float64, 5
    iterations) on the 12-component wide-spectrum mixture (eigenvalues
    log-uniform in [1e-3, 1]) with N_train reduced from 300,000 to 20,000 to
    keep the test short, 4,096 queries from the same mixture.  Score
    d log p / dy and d / dL_n of the hand-written backward against FP64
    central differences (h = 1e-4, <= 1e-4 relative) at d = 21, and against
    torch autograd through the functional restatement on a kernel subset."""
    from lakde_b200 import LocalKNearestKDE
    from lakde_b200.grad import log_pred_density
    from lakde_b200.synthetic import wide_spectrum_mixture

    Xn, Yn = wide_spectrum_mixture(seed=3, n_train=20_000, n_test=4_096, d=21)
    X = torch.tensor(Xn, dtype=torch.float64, device="cuda")
    Y = torch.tensor(Yn, dtype=torch.float64, device="cuda")
    m = LocalKNearestKDE(k_or_knn_graph=64, fused=True, cuda_graph=False)
    m.fit(X, iterations=5, sparsity_threshold=5e-4)
    W_triu, nu, _ = m.engine.posterior_factors()
    L = torch.linalg.inv(W_triu).mT.contiguous()  # L_n L_n^T = W_n^-1, lower
    L = torch.tril(L)
    D = X.shape[1]
    rng = np.random.default_rng(0)
    g = torch.tensor(rng.standard_normal(len(Y)) / 64, device="cuda")
    Yr = Y.clone().requires_grad_(True)
    Lr = L.clone().requires_grad_(True)
    (log_pred_density(X, Lr, nu, Yr) * g).sum().backward()
    f = lambda Lx, Yx: float((log_pred_density(X, Lx, nu, Yx) * g).sum())  # noqa: E731
    # kernels that carry weight: the nearest kernel of a few queries
    near = torch.cdist(Y[:64], X).argmin(1).cpu().numpy()
    h = 1e-4
    for t in range(8):
        q, d = int(rng.integers(len(Y))), int(rng.integers(D))
        e = torch.zeros_like(Y)
        e[q, d] = h
        fd = (f(L, Y + e) - f(L, Y - e)) / (2 * h)
        an = float(Yr.grad[q, d])
        assert abs(fd - an) <= 1e-4 * max(abs(an), 1e-3), ("score", q, d, fd, an)
        n = int(near[t])
        i = int(rng.integers(D))
        j = int(rng.integers(i + 1))
        e = torch.zeros_like(L)
        e[n, i, j] = h
        fd = (f(L + e, Y) - f(L - e, Y)) / (2 * h)
        an = float(Lr.grad[n, i, j])
        assert abs(fd - an) <= 1e-4 * max(abs(an), 1e-3), ("dL", n, i, j, fd, an)
    # torch autograd through the reference formula on 1,500 kernels x 512 queries
    sub, qs = slice(0, 1500), slice(0, 512)
    Xs, Ls, nus, Ys, gs = X[sub].cpu(), L[sub].cpu(), nu[sub].cpu(), Y[qs].cpu(), g[qs].cpu()
    Yt = Ys.clone().requires_grad_(True)
    Lt = Ls.clone().requires_grad_(True)
    (torch_reference(Xs, Lt, nus, Yt) * gs).sum().backward()
    Yc = Ys.cuda().requires_grad_(True)
    Lc = Ls.cuda().requires_grad_(True)
    (log_pred_density(Xs.cuda(), Lc, nus.cuda(), Yc) * gs.cuda()).sum().backward()
    torch.testing.assert_close(Yc.grad.cpu(), Yt.grad, rtol=1e-8, atol=1e-10)
    torch.testing.assert_close(Lc.grad.cpu(), torch.tril(Lt.grad), rtol=1e-8, atol=1e-10)
