"""The allocation-free predictive density entry point.

lakde_log_pred_density_noalloc serves callers that cannot call cudaMalloc
(hosts that own all device memory, or forbid allocation once running): its
scratch is an array built into the library instead of a caller workspace.
This checks it through the C ABI against lakde_log_pred_density on two calls
in a row, the second reusing the scratch left by the first.  The file is
named to be collected last.
"""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _case(rng, N, Nq, D, dtype):
    X = torch.tensor(rng.standard_normal((N, D)), dtype=dtype, device="cuda")
    Y = torch.tensor(rng.standard_normal((Nq, D)), dtype=dtype, device="cuda")
    W = np.triu(rng.standard_normal((N, D, D)) / np.sqrt(D))
    W[:, np.arange(D), np.arange(D)] = np.abs(W[:, np.arange(D), np.arange(D)]) + 0.5
    W = torch.tensor(W, dtype=dtype, device="cuda")
    nu = torch.tensor(rng.uniform(D + 1, D + 30, N), dtype=dtype, device="cuda")
    logdet = 2 * W.diagonal(dim1=1, dim2=2).log().sum(-1)
    return X, Y, W, nu, logdet


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_noalloc_matches_workspace_entry_point_on_consecutive_calls(dtype):
    from lakde_b200 import _native as nat
    from lakde_b200 import kernels as K

    lib = nat.lib()
    rng = np.random.default_rng(7)
    tol = 1e-6 if dtype == torch.float32 else 1e-12
    for N, Nq, D in ((3000, 1500, 8), (900, 4000, 21)):
        X, Y, W, nu, logdet = _case(rng, N, Nq, D, dtype)
        lc = K.pred_coeff(nu, logdet.contiguous(), D)
        ref = K.log_pred_density(X, W, nu, lc, Y)
        out = torch.full((Nq,), float("nan"), dtype=dtype, device="cuda")
        st = lib.lakde_log_pred_density_noalloc(
            nat.dtype_code(X), N, Nq, D, nat.ptr(X), nat.ptr(W), nat.ptr(nu), nat.ptr(lc), nat.ptr(Y), nat.ptr(out),
            nat.stream_of(out),
        )
        nat.check(st, "log_pred_density_noalloc")
        torch.cuda.synchronize()
        torch.testing.assert_close(out, ref, rtol=tol, atol=tol)


def test_noalloc_rejects_oversized_calls():
    from lakde_b200 import _native as nat

    lib = nat.lib()
    N, Nq, D = 10, 3_000_000, 2
    x = torch.zeros(16, device="cuda")
    st = lib.lakde_log_pred_density_noalloc(nat.F32, N, Nq, D, *(nat.ptr(x),) * 6, nat.stream_of(x))
    assert st == 1
    assert b"scratch" in lib.lakde_last_error()
