"""Host-side helpers of the VI path, mirroring lakde/utils.py.

compute_knn_graph ranks exact float64 distances on the GPU (a library GEMM
for the candidate distances, the library's selection kernel for the rest)
with a lower-index tie break (the order the oracle defines); batched_knn_cov
is the scatter-covariance kernel on the kNN rows.
"""

import signal

import torch

from . import kernels


def tensor_as(x, other):
    """lakde/utils.py:8-11."""
    if torch.is_tensor(x):
        return x.to(dtype=other.dtype, device=other.device)
    return torch.tensor(x, dtype=other.dtype, device=other.device)


def cov(X, dtype=None, inplace=False):
    """Unbiased sample covariance (lakde/utils.py:28-37)."""
    N = X.size(-2)
    if dtype is None:
        dtype = torch.promote_types(X.dtype, torch.float32)
    Xd = X.to(dtype)
    X_bar = Xd.mean(dim=-2, keepdim=True)
    Xc = Xd - X_bar
    return torch.matmul(Xc.mT, Xc).div_(N - 1)


def batched_knn_cov(X, X_self, knn_graph, include_self=False, self_center=True):
    """Sigma0[n] = 1/K sum_k (x_k - x_n)(x_k - x_n)^T over the kNN list of n.

    lakde/utils.py:40-65 with include_self=False, self_center=True (the only
    combination the locally adaptive models use), computed by the scatter
    kernel with weights 1/K on the rows of the graph.
    """
    if include_self or not self_center:
        raise NotImplementedError("only include_self=False, self_center=True is used by the models")
    M, K = knn_graph.shape
    rowptr = torch.arange(0, (M + 1) * K, K, device=X.device, dtype=torch.int64)
    col = knn_graph.reshape(-1).contiguous()
    w = torch.full((M * K,), 1.0 / K, dtype=X.dtype, device=X.device)
    return kernels.calc_W_inv(rowptr, col, w, X_self.contiguous(), X.contiguous())


def compute_knn_graph(X, k, bsize=1024, return_dists=False, include_self=False, metric="l2", dtype=torch.int32):
    """k nearest neighbours of every row of X, nearest first (lakde/utils.py:77-116).

    Per block of rows, one library GEMM gives the float64 squared distances
    |a|^2 + |b|^2 - 2ab to all points; lakde_knn_select (kernels.knn_select)
    keeps each row's k + 8 smallest in one pass, re-ranks them by exact
    float64 differences and writes the k nearest, equal distances ordered by
    index.
    """
    if metric.lower() != "l2":
        raise ValueError("only the l2 metric is supported")
    N = X.size(0)
    Xd = X.double().contiguous()
    sq = (Xd * Xd).sum(1)
    I = torch.empty(N, k, dtype=dtype, device=X.device)
    Dout = X.new_empty(N, k) if return_dists else None
    for i in range(0, N, bsize):
        Xb = Xd[i : i + bsize]
        d = torch.addmm(sq[None, :], Xb, Xd.T, alpha=-2.0).add_(sq[i : i + bsize, None])
        kernels.knn_select(d, Xd, i, k, include_self=include_self, out_idx=I[i : i + bsize],
                           out_dist=None if Dout is None else Dout[i : i + bsize])
    if return_dists:
        return Dout, I
    return I


class InterruptDelay:
    """Defers SIGINT while model state is being mutated (lakde/utils.py:240-255)."""

    def __init__(self):
        self.signal_received = None
        self.old_handler = None

    def __enter__(self):
        try:
            self.old_handler = signal.signal(signal.SIGINT, self._handler)
        except ValueError:  # not the main thread
            self.old_handler = None
        return self

    def _handler(self, sig, frame):
        print("Interrupt received during update, finishing up...")
        self.signal_received = (sig, frame)

    def __exit__(self, *exc):
        if self.old_handler is not None:
            signal.signal(signal.SIGINT, self.old_handler)
            if self.signal_received is not None and callable(self.old_handler):
                self.old_handler(*self.signal_received)
        return False
