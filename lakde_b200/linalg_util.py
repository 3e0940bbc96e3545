"""Numeric helpers of the VI path, mirroring lakde/linalg_util.py.

The per-kernel factorisations run in the FP64 CUDA kernel
(``kernels.posterior_factor``); the small scalar helpers are torch
expressions evaluated on the device of their inputs.
"""

import math

import torch

from . import kernels


def lgamma(a):
    """log Gamma evaluated in float64 and cast back (lakde/linalg_util.py:8-9)."""
    return torch.lgamma(a.double()).to(a.dtype)


def mvlgamma(a, D):
    """Multivariate log Gamma (lakde/linalg_util.py:13-18)."""
    i = torch.arange(1, D + 1, dtype=a.dtype, device=a.device)
    terms = lgamma(a.unsqueeze(-1) + (1 - i) / 2)
    return D * (D - 1) / 4 * math.log(math.pi) + terms.sum(-1)


def mvdigamma(a, D):
    """sum_{i=1..D} psi(a + (1 - i)/2) (lakde/linalg_util.py:22-26)."""
    i = torch.arange(1, D + 1, dtype=a.dtype, device=a.device)
    return torch.digamma(a.unsqueeze(-1) + (1 - i) / 2).sum(-1)


def chol_logdet(L):
    """2 sum log diag(L) (lakde/linalg_util.py:30-31)."""
    return 2 * L.diagonal(dim1=-2, dim2=-1).log().sum(dim=-1)


def chol_mm_trace(L, R):
    """||L^T R||_F^2 (lakde/linalg_util.py:35-37)."""
    LR = L.mT @ R
    return LR.pow_(2).sum(dim=(-1, -2))


def logsubexp(a, b):
    """a + log1p(max(-exp(b - a), -1)) (lakde/linalg_util.py:41-42)."""
    return a + torch.log1p(torch.clamp_min(-torch.exp(b - a), -1))


def xlogx(x, out=None):
    return torch.xlogy(x, x, out=out)


def tril_inverse(L):
    """Inverse of a lower-triangular matrix (lakde/linalg_util.py:49-52)."""
    D = L.size(-1)
    eye = torch.eye(D, dtype=L.dtype, device=L.device).expand_as(L).contiguous()
    return torch.linalg.solve_triangular(L, eye, upper=False)


def stabilized_cholesky(X, jitter=None, out=None, verbose=False):
    """Jittered Cholesky with the per-matrix eps * 2^k ladder (lakde/linalg_util.py:129-170).

    Runs in the FP64 CUDA kernel; the ladder is evaluated on the device per
    matrix.  Returns (L, jitter) like the reference; raises RuntimeError
    ("Stabilization did not converge") when a matrix stays indefinite after 32
    doublings.  ``jitter`` is returned as a new tensor (or None if it was None
    and no matrix needed one).
    """
    single = X.dim() == 2
    Xb = X.unsqueeze(0) if single else X
    N = Xb.size(0)
    jit = Xb.new_zeros(N) if jitter is None else jitter.reshape(N).clone()
    eps = torch.finfo(X.dtype).eps
    _, _, info, L, _ = kernels.posterior_factor(Xb.contiguous(), jit, eps, want_L=True)
    if bool((info != 0).any()):
        raise RuntimeError("Stabilization did not converge")
    if verbose and bool((jit != (0 if jitter is None else jitter.reshape(N))).any()):
        print("Found new jitter values {}".format(jit[jit != 0]))
    if single:
        L = L[0]
        jit = jit.reshape(())
    if jitter is None and not bool((jit != 0).any()):
        jit = None
    if out is not None:
        out.copy_(L)
        L = out
    return L, jit
