"""Differentiable predictive log density.

``log_pred_density(X, L, nu, Y)`` evaluates the Student-t mixture of
lakde/local_adaptive_kde.py:200-223 from the kernels' Cholesky factors
``L_n`` (lower, ``L_n L_n^T = W_n^-1``) and returns a tensor whose backward is
the hand-written CUDA pass of ``kernels.log_pred_density_bwd``: gradients for
the queries ``Y`` (the score d log p(y) / dy) and for the factors ``L``.
The reference's own log_pred_density is not differentiable (it accumulates
with ``torch.logaddexp(..., out=)``).
"""

import torch

from . import kernels as K


def _upper_inverse_t(L):
    """W_triu = L^-T for a batch of lower-triangular factors."""
    D = L.size(-1)
    eye = torch.eye(D, dtype=L.dtype, device=L.device).expand_as(L)
    return torch.linalg.solve_triangular(L, eye, upper=False).mT.contiguous()


class _LogPredDensity(torch.autograd.Function):
    @staticmethod
    def forward(ctx, Y, L, X, nu):
        D = X.size(1)
        U = _upper_inverse_t(L)
        logdet = (-2 * torch.log(torch.diagonal(L, dim1=-2, dim2=-1)).sum(-1)).contiguous()
        lc = K.pred_coeff(nu.contiguous(), logdet, D)
        out = K.log_pred_density(X.contiguous(), U, nu.contiguous(), lc, Y)
        ctx.save_for_backward(Y, L, X, nu, U, lc, out)
        return out

    @staticmethod
    def backward(ctx, g):
        Y, L, X, nu, U, lc, out = ctx.saved_tensors
        gY, sw, S_c = K.log_pred_density_bwd(X.contiguous(), U, nu.contiguous(), lc, Y, out, g)
        gL = None
        if ctx.needs_input_grad[1]:
            h = (nu + 1) / 2
            M = U.mT @ S_c @ U  # sum_y c_ny z z^T
            gL = (2 * h)[:, None, None] * (U @ M)
            gL.diagonal(dim1=-2, dim2=-1).sub_(sw[:, None] / torch.diagonal(L, dim1=-2, dim2=-1))
            gL = torch.tril(gL)
        return (gY if ctx.needs_input_grad[0] else None), gL, None, None


def log_pred_density(X, L, nu, Y):
    """log p(Y) under the mixture with kernel centres X [N, D], Cholesky
    factors L [N, D, D] of W^-1 and degrees of freedom nu [N]; differentiable
    in Y and L."""
    return _LogPredDensity.apply(Y, L, X, nu)
