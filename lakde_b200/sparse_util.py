"""Responsibility-pattern layouts, mirroring lakde/sparse_util.py.

The reference stores responsibilities per kernel block as COO (row = kernel n
relative to the block, col = point m) sorted by row
(lakde/sparse_util.py:8-54).  The fused path keeps one fixed pair pattern for
all kernels in CSR form grouped by kernel, plus a point-major permutation for
the per-point normaliser (``PairPattern``).
"""

import itertools

import torch

from . import kernels


def _ind2ptr(row, M):
    out = torch.empty(M + 1, dtype=torch.int64, device=row.device)
    return kernels.ind2ptr(row.contiguous(), M, out=out)


def graph_to_slices(graph, block_size):
    """Per-block COO [2, nnz_b] pattern of (n in kNN(m), m), sorted by (row, col).

    lakde/sparse_util.py:40-54; within a row the columns are ascending (the
    reference leaves that order to an unstable argsort).
    """
    N, K = graph.shape
    rows = graph.reshape(-1).long()
    cols = torch.arange(N, device=graph.device).repeat_interleave(K)
    order = torch.argsort(rows * N + cols)
    rows, cols = rows[order], cols[order]
    ptr = _ind2ptr(rows, N).cpu()
    out = []
    for s in range(0, N, block_size):
        e = min(s + block_size, N)
        a, b = int(ptr[s]), int(ptr[e])
        out.append(torch.stack((rows[a:b] - s, cols[a:b])).to(graph.dtype))
    return out


def cat_sparse(all_indices, all_values, shifts, dim=0):
    """lakde/sparse_util.py:57-71."""
    offset = 0
    shifted = []
    if isinstance(shifts, int):
        shifts = itertools.repeat(shifts)
    for inds, shift in zip(all_indices, shifts):
        inds = inds.clone()
        inds[dim] += offset
        shifted.append(inds)
        offset += shift
    if all_values is not None:
        return torch.cat(shifted, dim=1), torch.cat(all_values)
    return torch.cat(shifted, dim=1)


class PairPattern:
    """A fixed set of (kernel n, point m) pairs.

    Kernel-major CSR: pairs of kernel n are ``col[rowptr[n]:rowptr[n+1]]``
    (ascending m).  Point-major view: the CSR positions of the pairs of point m
    are ``pos[cptr[m]:cptr[m+1]]`` (ascending n).  ``rank`` optionally keeps,
    per pair, the position of n in the candidate list of m (used to seed the
    initial responsibilities).
    """

    def __init__(self, rowptr, col, cptr, pos, n_kernels, n_points, rank=None):
        self.rowptr = rowptr
        self.col = col
        self.cptr = cptr
        self.pos = pos
        self.n_kernels = n_kernels
        self.n_points = n_points
        self.rank = rank
        # kernel rows longest first: the fused per-row kernel walks rows in this
        # order so the threads of a warp carry rows of similar length
        lengths = rowptr[1:] - rowptr[:-1]
        self.order = torch.argsort(lengths, descending=True, stable=True).to(torch.int32)

    @property
    def nnz(self):
        return self.col.numel()

    @property
    def device(self):
        return self.col.device

    @classmethod
    def from_pairs(cls, kern, point, n_kernels, n_points, rank=None):
        kern = kern.long()
        point = point.long()
        order = torch.argsort(kern * n_points + point)
        k_s, p_s = kern[order], point[order]
        rowptr = _ind2ptr(k_s, n_kernels)
        col = p_s.to(torch.int32)
        pos = torch.argsort(p_s * n_kernels + k_s)
        cptr = _ind2ptr(p_s[pos], n_points)
        pos = pos.to(torch.int32) if p_s.numel() < 2**31 else pos
        return cls(rowptr, col, cptr, pos, n_kernels, n_points, None if rank is None else rank[order])

    @classmethod
    def from_knn_graph(cls, graph):
        """Pairs (graph[m, k], m): kernel n explains point m when n is one of its
        K nearest neighbours -- the pattern the reference seeds its
        responsibilities with (lakde/sparse_util.py:8-17, lakde/local_knn_kde.py:113-127)."""
        N, K = graph.shape
        kern = graph.reshape(-1)
        point = torch.arange(N, device=graph.device).repeat_interleave(K)
        rank = torch.arange(K, device=graph.device, dtype=torch.int32).repeat(N)
        return cls.from_pairs(kern, point, N, N, rank)

    @classmethod
    def from_knn_counts(cls, graph, counts):
        """Uneven neighbourhoods: point m is explained by its first counts[m]
        nearest kernels graph[m, :counts[m]] (graph [N, Kmax], counts <= Kmax)."""
        N, Kmax = graph.shape
        counts = torch.as_tensor(counts, device=graph.device).long().clamp(0, Kmax)
        keep = torch.arange(Kmax, device=graph.device)[None, :] < counts[:, None]
        kern = graph.long()[keep]
        point = torch.arange(N, device=graph.device).repeat_interleave(counts)
        return cls.from_pairs(kern, point, N, N)

    @classmethod
    def from_neighbour_lists(cls, graph, counts):
        """Variable-length candidate lists: the first counts[m] entries of graph[m]."""
        N, K = graph.shape
        counts = counts.to(graph.device).clamp(max=K)
        keep = torch.arange(K, device=graph.device)[None, :] < counts[:, None]
        kern = graph[keep]
        point = torch.arange(N, device=graph.device)[:, None].expand(N, K)[keep]
        rank = torch.arange(K, device=graph.device, dtype=torch.int32)[None, :].expand(N, K)[keep]
        return cls.from_pairs(kern, point, N, N, rank)

    @classmethod
    def dense(cls, N, device):
        """Every pair (n, m), n != m included as -inf by the E-step: the
        pattern of the reference's dense E-step."""
        idx = torch.arange(N, device=device)
        kern = idx.repeat_interleave(N)
        point = idx.repeat(N)
        return cls.from_pairs(kern, point, N, N)

    def rows(self):
        """Kernel index of every pair (CSR order)."""
        counts = self.rowptr[1:] - self.rowptr[:-1]
        return torch.repeat_interleave(torch.arange(self.n_kernels, device=self.device), counts)

    def to_blocks(self, values, block_size):
        """Reference-layout COO blocks [(indices [2, nnz_b] int32, values)],
        keeping only non-zero values (lakde/local_adaptive_kde.py:140-150)."""
        rows = self.rows()
        cols = self.col.long()
        keep = values != 0
        rows, cols, values = rows[keep], cols[keep], values[keep]
        ptr = _ind2ptr(rows, self.n_kernels).cpu()
        out = []
        for s in range(0, self.n_kernels, block_size):
            e = min(s + block_size, self.n_kernels)
            a, b = int(ptr[s]), int(ptr[e])
            out.append((torch.stack((rows[a:b] - s, cols[a:b])).to(torch.int32), values[a:b]))
        return out
