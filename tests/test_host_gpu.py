"""Host-side GPU helpers against the oracle: the kNN graph (bit-exact order
under exact float64 distances with index tie-break), the reference COO layout
and the pair pattern."""

import numpy as np
import pytest
import torch

from oracle import lakde_oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("include_self", [False, True])
@pytest.mark.parametrize("N,D,k", [(700, 3, 10), (3000, 8, 50), (2500, 43, 30), (3000, 6, 600), (4100, 5, 1500)])
def test_knn_graph_is_exact(N, D, k, include_self):
    from lakde_b200.utils import compute_knn_graph

    rng = np.random.default_rng(N + D)
    X = rng.standard_normal((N, D)).astype(np.float32)
    X[5] = X[9]  # an exact duplicate: tie broken by index
    g = compute_knn_graph(torch.tensor(X, device="cuda"), k, bsize=512, include_self=include_self)
    np.testing.assert_array_equal(g.cpu().numpy(), O.knn_graph(X, k, include_self=include_self))


@pytest.mark.parametrize("out_dtype", [torch.float32, torch.float64])
def test_knn_graph_distances_and_index_dtype(out_dtype):
    from lakde_b200.utils import compute_knn_graph

    rng = np.random.default_rng(7)
    X = rng.standard_normal((1500, 7)).astype(np.float32)
    Xt = torch.tensor(X, device="cuda").to(out_dtype)
    d, g = compute_knn_graph(Xt, 20, bsize=256, return_dists=True, dtype=torch.int64)
    assert g.dtype == torch.int64 and d.dtype == out_dtype
    g = g.cpu().numpy()
    np.testing.assert_array_equal(g, O.knn_graph(X, 20))
    X64 = X.astype(np.float64)
    exact = np.sqrt(((X64[g] - X64[:, None, :]) ** 2).sum(-1))
    np.testing.assert_allclose(d.cpu().numpy(), exact, rtol=1e-6 if out_dtype == torch.float32 else 1e-12)


def test_pattern_views_are_consistent():
    from lakde_b200.sparse_util import PairPattern, graph_to_slices

    rng = np.random.default_rng(0)
    X = rng.standard_normal((600, 4)).astype(np.float32)
    graph = O.knn_graph(X, 9)
    pat = PairPattern.from_knn_graph(torch.tensor(graph, device="cuda"))
    rows = pat.rows().cpu().numpy()
    col = pat.col.cpu().numpy()
    ref = O.knn_pattern(graph)[0]
    np.testing.assert_array_equal(rows, ref[0])
    np.testing.assert_array_equal(col, ref[1])
    # point-major view lists, for each point, its pairs in ascending kernel order
    pos = pat.pos.long().cpu().numpy()
    cptr = pat.cptr.cpu().numpy()
    for m in (0, 17, 599):
        p = pos[cptr[m] : cptr[m + 1]]
        assert (col[p] == m).all()
        np.testing.assert_array_equal(np.sort(rows[p]), np.sort(graph[m]))
        assert (np.diff(rows[p]) > 0).all()
    blocks = graph_to_slices(torch.tensor(graph, device="cuda"), 128)
    for bi, b in enumerate(blocks):
        np.testing.assert_array_equal(b.cpu().numpy(), O.knn_pattern(graph, 128)[bi])
