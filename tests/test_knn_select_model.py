"""A model of the selection pass of lakde_b200/csrc/knn.cu (knn_select_kernel):
one streaming pass over a row of distances in chunks of 1,024, values below
a running threshold appended to a buffer of `cap` entries, the buffer sorted
by (value, index) and cut to its kc smallest whenever the next chunk could
overflow it, the kc-th value becoming the threshold.  The kernel's
candidates are the first kc entries of the final sort.

The model checks the design on adversarial orders (descending values force
a cut at every chunk), ties and NaN: the candidates must be exactly the kc
smallest by (value, index), which the exact re-ranking then orders.  The GPU
tests check the compiled kernel against the oracle."""

import numpy as np
import pytest

CHUNK = 1024


def cap_for(kc):
    cap = 2048
    while cap < kc + CHUNK:
        cap *= 2
    return cap


def select_model(row, kc, self_idx=None):
    """The kernel's candidate set for one row: list of (value, index)."""
    N = len(row)
    cap = cap_for(kc)
    buf = []
    thr = np.inf
    cuts = 0
    for base in range(0, N, CHUNK):
        if len(buf) + CHUNK > cap:
            buf.sort()
            buf = buf[:kc]
            thr = buf[-1][0]
            cuts += 1
        for j in range(base, min(base + CHUNK, N)):
            v = row[j]
            if np.isnan(v) or j == self_idx:
                v = np.inf
            if v < thr:
                buf.append((v, j))
                assert len(buf) <= cap, "buffer overflow"
    buf.sort()
    return buf[:kc], cuts


def expected(row, kc, self_idx=None):
    v = np.where(np.isnan(row), np.inf, row).astype(np.float64)
    if self_idx is not None:
        v[self_idx] = np.inf
    order = np.lexsort((np.arange(len(v)), v))
    return [(v[i], int(i)) for i in order[:kc]]


@pytest.mark.parametrize("order", ["random", "descending", "ascending", "ties"])
@pytest.mark.parametrize("N,kc", [(700, 18), (5000, 108), (20000, 108), (12000, 1508), (9000, 4104)])
def test_candidates_are_the_kc_smallest(order, N, kc):
    if kc > N - 1:
        pytest.skip("more candidates than points")
    rng = np.random.default_rng(N + kc)
    row = rng.standard_normal(N)
    if order == "descending":
        row = np.sort(row)[::-1].copy()
    elif order == "ascending":
        row = np.sort(row)
    elif order == "ties":
        row = np.round(row, 1)  # a few dozen distinct values, ties everywhere
    self_idx = N // 3
    got, cuts = select_model(row, kc, self_idx)
    assert got == expected(row, kc, self_idx)
    if order == "descending" and N > cap_for(kc):
        assert cuts > 0


def test_nan_and_self_never_become_candidates():
    rng = np.random.default_rng(3)
    row = rng.standard_normal(6000)
    row[::7] = np.nan
    got, _ = select_model(row, 50, self_idx=11)
    assert all(np.isfinite(v) for v, _ in got) and all(j != 11 for _, j in got)
    assert got == expected(row, 50, 11)
