"""Drop-in replacement for lakde/kernels.py backed by the sm_100a library.

The three custom ops keep the reference schemas in the ``lakde`` namespace
(csrc/cuda/convert_cuda.cu:67-68, W_inv_cuda.cu:139-140,
chol_quad_form.cu:116-117):

    lakde::ind2ptr_cuda(Tensor ind, int M, Tensor out) -> Tensor
    lakde::W_inv_cuda(Tensor rowptr, Tensor col, Tensor value, Tensor Xn, Tensor Xm, Tensor out) -> Tensor
    lakde::chol_quad_form_cuda(Tensor W_triu, Tensor Xn, Tensor Xm, Tensor out) -> Tensor

and the Python wrappers ``ind2ptr``, ``calc_W_inv`` and ``chol_quad_form``
keep the signatures of lakde/kernels.py:93-120.  The caller-visible
difference: tensors on the CPU are rejected with an error instead of being
routed to the slow torch fallbacks; the ops run only on the GPU.  float16
values are not supported (float32 and float64 are).

The new ops of the fused path (posterior factorisation, sparse E-step,
normaliser, predictive density) are exposed as functions below; each maps
one-to-one onto an entry point of include/lakde_b200.h.
"""

import torch

from . import _native as nat

_LIB = torch.library.Library("lakde", "DEF")
_LIB.define("ind2ptr_cuda(Tensor ind, int M, Tensor out) -> Tensor")
_LIB.define("W_inv_cuda(Tensor rowptr, Tensor col, Tensor value, Tensor Xn, Tensor Xm, Tensor out) -> Tensor")
_LIB.define("chol_quad_form_cuda(Tensor W_triu, Tensor Xn, Tensor Xm, Tensor out) -> Tensor")


def _assert(cond, msg="Input mismatch"):
    if not cond:
        raise RuntimeError(msg)


def _ind2ptr_cuda(ind, M, out):
    nat.require_cuda(ind, out, op="ind2ptr_cuda")
    _assert(ind.dim() == 1 and ind.is_contiguous(), "ind must be a contiguous 1-d tensor")
    _assert(out.dim() == 1 and out.numel() == M + 1 and out.is_contiguous(), "out must be contiguous with M + 1 entries")
    lib = nat.lib()
    nat.check(
        lib.lakde_ind2ptr(
            nat.ptr(ind), nat.dtype_code(ind), ind.numel(), M, nat.ptr(out), nat.dtype_code(out), nat.stream_of(out)
        ),
        "ind2ptr_cuda",
    )
    return out


def _W_inv_cuda(rowptr, col, value, Xn, Xm, out):
    nat.require_cuda(rowptr, col, value, Xn, Xm, out, op="W_inv_cuda")
    _assert(rowptr.dim() == 1)
    _assert(col.dim() == 1)
    _assert(value.size(0) == col.size(0))
    _assert(value.dim() == 1)
    _assert(Xn.dim() == 2)
    _assert(Xm.dim() == 2)
    N, D = Xn.shape
    _assert(rowptr.numel() - 1 == N)
    _assert(Xm.size(1) == D)
    _assert(Xn.is_contiguous() and Xm.is_contiguous() and out.is_contiguous())
    _assert(rowptr.is_contiguous() and col.is_contiguous() and value.is_contiguous())
    _assert(out.shape == (N, D, D), "out must have shape [N, D, D]")
    _assert(value.dtype == Xn.dtype == Xm.dtype == out.dtype, "value, Xn, Xm and out must share a dtype")
    nat.check(
        nat.lib().lakde_W_inv(
            nat.dtype_code(value),
            nat.ptr(rowptr),
            nat.dtype_code(rowptr),
            nat.ptr(col),
            nat.dtype_code(col),
            nat.ptr(value),
            nat.ptr(Xn),
            nat.ptr(Xm),
            nat.ptr(out),
            N,
            Xm.size(0),
            D,
            nat.stream_of(out),
        ),
        "W_inv_cuda",
    )
    return out


def _chol_quad_form_cuda(W_triu, Xn, Xm, out):
    nat.require_cuda(W_triu, Xn, Xm, out, op="chol_quad_form_cuda")
    _assert(W_triu.dim() == 3)
    _assert(Xn.dim() == 2)
    _assert(Xm.dim() == 2)
    N, M, D = Xn.size(0), Xm.size(0), Xn.size(1)
    _assert(Xm.size(1) == D)
    _assert(W_triu.size(0) == N)
    _assert(W_triu.size(1) == D)
    _assert(W_triu.size(2) == D)
    _assert(out.dim() == 2 and out.size(0) == N and out.size(1) == M, "out must have shape [N, M]")
    _assert(W_triu.dtype == Xn.dtype == Xm.dtype == out.dtype, "all tensors must share a dtype")
    nat.check(
        nat.lib().lakde_chol_quad_form(
            nat.dtype_code(W_triu),
            nat.ptr(W_triu),
            nat.strides(W_triu),
            nat.ptr(Xn),
            nat.strides(Xn),
            nat.ptr(Xm),
            nat.strides(Xm),
            nat.ptr(out),
            nat.strides(out),
            N,
            M,
            D,
            nat.stream_of(out),
        ),
        "chol_quad_form_cuda",
    )
    return out


_LIB.impl("ind2ptr_cuda", _ind2ptr_cuda, "CUDA")
_LIB.impl("W_inv_cuda", _W_inv_cuda, "CUDA")
_LIB.impl("chol_quad_form_cuda", _chol_quad_form_cuda, "CUDA")


# --------------------------------------------------------------------------
# Python wrappers with the reference signatures (lakde/kernels.py:93-120)
# --------------------------------------------------------------------------


def ind2ptr(ind, M, out=None):
    assert ind.is_contiguous()
    if out is None:
        out = ind.new_empty(M + 1)
    nat.require_cuda(ind, op="ind2ptr")
    return torch.ops.lakde.ind2ptr_cuda(ind, M, out)


def calc_W_inv(rowptr, col, value, Xn, Xm):
    assert rowptr.is_contiguous()
    assert col.is_contiguous()
    assert value.is_contiguous()
    assert Xn.is_contiguous()
    assert Xm.is_contiguous()
    nat.require_cuda(rowptr, op="calc_W_inv")
    N, D = Xn.shape
    out = value.new_empty(N, D, D)
    return torch.ops.lakde.W_inv_cuda(rowptr, col, value, Xn, Xm, out)


def chol_quad_form(W_triu, Xn, Xm):
    nat.require_cuda(W_triu, op="chol_quad_form")
    out = W_triu.new_empty(Xn.size(0), Xm.size(0))
    return torch.ops.lakde.chol_quad_form_cuda(W_triu, Xn, Xm, out)


# --------------------------------------------------------------------------
# New ops of the hot path
# --------------------------------------------------------------------------


def mstep(rowptr, col, r, X, nu_0, kernel_offset=0, S=None, nu=None):
    """Scatter covariance S and nu = nu_0 + row sums of r for kernels kernel_offset.. of X."""
    nat.require_cuda(rowptr, col, r, X, op="mstep")
    N = rowptr.numel() - 1
    D = X.size(1)
    S = X.new_empty(N, D, D) if S is None else S
    nu = X.new_empty(N) if nu is None else nu
    nat.check(
        nat.lib().lakde_mstep(
            nat.dtype_code(X), N, D, X.size(0), nat.ptr(rowptr), nat.dtype_code(rowptr), nat.ptr(col),
            nat.dtype_code(col), nat.ptr(r), nat.ptr(X), kernel_offset, float(nu_0), nat.ptr(S), nat.ptr(nu),
            nat.stream_of(X),
        ),
        "mstep",
    )
    return S, nu


def posterior_factor(S, jitter, eps, P=None, nu_0=None, a=None, b=None, T=None, want_L=False, info=None, out=None,
                     logdet=None, trace=None, L=None, T_lower=False, W_cores=None):
    """FP64 jittered Cholesky of A_n = nu_0 a_n / b_n P_n + S_n (see include/lakde_b200.h).

    Returns (W_triu, logdet_W, info, L or None, trace or None); ``jitter`` is
    updated in place.  ``P`` and ``T`` may be [D, D] (shared) or [N, D, D].
    Output buffers may be passed in (out, logdet, info, trace, L).
    ``T_lower=True`` declares T lower triangular (its upper part is not read).
    ``W_cores`` (float32, from ``w_cores_like``) also receives W_triu as the
    tensor-core kernels' W cores.
    """
    nat.require_cuda(S, jitter, P, nu_0, a, b, T, op="posterior_factor")
    N, D, _ = S.shape
    S = S.contiguous()
    dt = S.dtype
    W = torch.empty_like(S) if out is None else out
    logdet = S.new_empty(N) if logdet is None else logdet
    info = S.new_empty(N, dtype=torch.int32) if info is None else info
    if L is None and want_L:
        L = torch.empty_like(S)
    if T is not None and trace is None:
        trace = S.new_empty(N)

    def batch(M):
        if M is None:
            return None, 0
        M = M.to(dt).contiguous()
        return M, (0 if M.dim() == 2 else D * D)

    P, pbs = batch(P)
    T, tbs = batch(T)
    if nu_0 is not None:
        nu_0 = nu_0.to(dt).reshape(1).contiguous()
    if a is not None:
        a = a.to(dt).contiguous()
        b = b.to(dt).contiguous()
    assert jitter.dtype == dt and jitter.is_contiguous() and jitter.numel() == N
    nat.check(
        nat.lib().lakde_posterior_factor(
            nat.dtype_code(S), N, D, nat.ptr(S), nat.ptr(P), pbs, nat.ptr(nu_0), nat.ptr(a), nat.ptr(b),
            nat.ptr(jitter), float(eps), nat.ptr(W), nat.ptr(L), nat.ptr(logdet), nat.ptr(info), nat.ptr(T), tbs,
            int(bool(T_lower)), nat.ptr(trace), nat.ptr(W_cores), nat.stream_of(S),
        ),
        "posterior_factor",
    )
    return W, logdet, info, L, trace


def estep_logrho(rowptr, col, X, W_triu, nu, logdet_W, kernel_offset=0, out=None):
    """log rho for every pair of a kernel-major CSR pattern (see include/lakde_b200.h)."""
    nat.require_cuda(rowptr, col, X, W_triu, nu, logdet_W, op="estep_logrho")
    N = rowptr.numel() - 1
    D = X.size(1)
    out = X.new_empty(col.numel()) if out is None else out
    nat.check(
        nat.lib().lakde_estep_logrho(
            nat.dtype_code(X), N, D, X.size(0), nat.ptr(rowptr), nat.dtype_code(rowptr), nat.ptr(col),
            nat.dtype_code(col), nat.ptr(X), kernel_offset, nat.ptr(W_triu), nat.ptr(nu), nat.ptr(logdet_W),
            nat.ptr(out), nat.stream_of(X),
        ),
        "estep_logrho",
    )
    return out


def vi_rows(rowptr, col, r, X, nu_0, a, b, b_0, jitter, eps, nu, logdet_W, info, logrho, P=None, T=None,
            order=None, mm=None, kernel_offset=0):
    """Fused per-kernel pass of one VI iteration, one thread per kernel row,
    D <= 8 (lakde_vi_rows, see include/lakde_b200.h).  Row n is the kernel
    centred on X[n + kernel_offset] (a shard's rows)."""
    nat.require_cuda(rowptr, col, r, X, a, b, jitter, nu, logdet_W, info, logrho, P, T, order, mm, op="vi_rows")
    entry = nat.lib().lakde_vi_rows
    N = rowptr.numel() - 1
    D = X.size(1)
    assert rowptr.dtype == torch.int64 and col.dtype == torch.int32
    assert order is None or order.dtype == torch.int32
    pbs = 0 if P is None or P.dim() == 2 else D * D
    tbs = 0 if T is None or T.dim() == 2 else D * D
    nat.check(
        entry(
            nat.dtype_code(X), N, D, X.size(0), nat.ptr(rowptr), nat.ptr(col), nat.ptr(order), nat.ptr(r),
            nat.ptr(X), int(kernel_offset), float(nu_0), nat.ptr(P), pbs, nat.ptr(T), tbs, nat.ptr(a), nat.ptr(b),
            float(b_0),
            nat.ptr(jitter), float(eps), nat.ptr(nu), nat.ptr(logdet_W), nat.ptr(mm), nat.ptr(info), nat.ptr(logrho),
            nat.stream_of(X),
        ),
        "vi_rows",
    )


def estep_normalise(cptr, pos, logrho, r, c, rsum, mode, threshold):
    """Per-point normaliser, responsibilities and rebalance (see include/lakde_b200.h)."""
    nat.require_cuda(cptr, pos, logrho, r, c, rsum, op="estep_normalise")
    assert cptr.dtype == torch.int64
    nat.check(
        nat.lib().lakde_estep_normalise(
            nat.dtype_code(logrho), c.numel(), nat.ptr(cptr), nat.ptr(pos), nat.dtype_code(pos), nat.ptr(logrho),
            nat.ptr(r), nat.ptr(c), nat.ptr(rsum), int(mode), float(threshold or 0.0), nat.stream_of(c),
        ),
        "estep_normalise",
    )


def estep_normalise_stage(stage, cptr, pos, logrho, r, c, rsum, red, red2, mode, threshold):
    """One stage of the per-point pass for kernels sharded over devices (see
    include/lakde_b200.h); the caller reduces red / red2 / rsum between stages."""
    nat.require_cuda(cptr, pos, logrho, r, c, rsum, red, red2, op="estep_normalise_stage")
    assert cptr.dtype == torch.int64
    nat.check(
        nat.lib().lakde_estep_normalise_stage(
            nat.dtype_code(c), int(stage), c.numel(), nat.ptr(cptr), nat.ptr(pos), nat.dtype_code(pos),
            nat.ptr(logrho), nat.ptr(r), nat.ptr(c), nat.ptr(rsum), nat.ptr(red), nat.ptr(red2), int(mode),
            float(threshold or 0.0), nat.stream_of(c),
        ),
        "estep_normalise_stage",
    )


def pred_coeff(nu, logdet_W, D, out=None):
    nat.require_cuda(nu, logdet_W, op="pred_coeff")
    out = torch.empty_like(nu) if out is None else out
    nat.check(
        nat.lib().lakde_pred_coeff(
            nat.dtype_code(nu), nu.numel(), D, nat.ptr(nu), nat.ptr(logdet_W), nat.ptr(out), nat.stream_of(nu)
        ),
        "pred_coeff",
    )
    return out


def log_pred_density_workspace_bytes(dtype, N, Nq, D):
    return int(nat.lib().lakde_log_pred_density_workspace(nat._DTYPE_CODES[dtype], N, Nq, D))


def log_pred_density(X, W_triu, nu, log_coeff, Y, out=None, workspace=None):
    """Student-t mixture log density of the rows of Y (see include/lakde_b200.h)."""
    nat.require_cuda(X, W_triu, nu, log_coeff, Y, op="log_pred_density")
    N, D = X.shape
    Y = Y.contiguous()
    Nq = Y.size(0)
    out = Y.new_empty(Nq) if out is None else out
    if Nq == 0:
        return out
    need = log_pred_density_workspace_bytes(X.dtype, N, Nq, D)
    if workspace is None or workspace.numel() < need:
        workspace = torch.empty(need, dtype=torch.uint8, device=X.device)
    nat.check(
        nat.lib().lakde_log_pred_density(
            nat.dtype_code(X), N, Nq, D, nat.ptr(X), nat.ptr(W_triu), nat.ptr(nu), nat.ptr(log_coeff),
            nat.ptr(Y), nat.ptr(out), nat.ptr(workspace), workspace.numel(), nat.stream_of(X),
        ),
        "log_pred_density",
    )
    return out


def tile_count(D):
    """Number of lower 8 x 8 tiles of the tiled layout for dimension D (see include/lakde_b200.h)."""
    return int(nat.lib().lakde_tile_count(int(D)))


def pack_tiles(src, dst, dst_tile_stride, dst_offset):
    """Lower tiles of src [N, D, D] into dst [N, tiles * dst_tile_stride] at dst_offset within each tile slot."""
    nat.require_cuda(src, dst, op="pack_tiles")
    N, D, _ = src.shape
    src = src.contiguous()
    assert dst.dtype == src.dtype and dst.is_contiguous() and dst.size(0) == N
    nat.check(
        nat.lib().lakde_pack_tiles(nat.dtype_code(src), N, D, nat.ptr(src), D * D, nat.ptr(dst), dst.stride(0),
                                   int(dst_tile_stride), int(dst_offset), nat.stream_of(src)),
        "pack_tiles",
    )
    return dst


def rows16(X):
    """(tensor, row stride) with 16-byte aligned rows for the tensor-core kernels:
    X itself when its rows already are (contiguous columns, a row stride that is
    a multiple of 4 floats, an aligned base), else a zero-padded copy."""
    D = X.size(1)
    if (X.stride(1) == 1 and X.stride(0) % 4 == 0 and X.stride(0) >= ((D + 3) // 4) * 4
            and X.data_ptr() % 16 == 0):
        return X, X.stride(0)
    Xp = pad_rows(X)
    return Xp, Xp.stride(0)


def pad_rows(X, out=None):
    """X [n, D] copied into the first D columns of a zero-padded [n, D rounded up
    to 4] buffer (returned as that view); ``out`` reuses such a buffer."""
    n, D = X.shape
    if out is None:
        out = X.new_zeros(n, ((D + 3) // 4) * 4)[:, :D]
    out.copy_(X)
    return out


def w_cores_like(D, N, device):
    """Buffer for the W cores of N kernels (float32; layout at lakde_pack_w_cores)."""
    return torch.empty(N, int(nat.lib().lakde_w_cores_floats(int(D))), dtype=torch.float32, device=device)


def pack_w_cores(W_triu, out=None):
    """W cores of W_triu [N, D, D] (dense upper triangles, float32)."""
    nat.require_cuda(W_triu, out, op="pack_w_cores")
    N, D, _ = W_triu.shape
    W_triu = W_triu.contiguous()
    out = w_cores_like(D, N, W_triu.device) if out is None else out
    nat.check(nat.lib().lakde_pack_w_cores(nat.dtype_code(W_triu), N, D, nat.ptr(W_triu), nat.ptr(out),
                                           nat.stream_of(W_triu)), "pack_w_cores")
    return out


def mstep_tc_tiled(rowptr, col, r, X, nu_0, err, SP, nu, order=None, kernel_offset=0, queue=None):
    """Tensor-core M-step writing S_n as tiles into the S halves of SP (see include/lakde_b200.h)."""
    nat.require_cuda(rowptr, col, r, X, err, SP, nu, order, queue, op="mstep_tc_tiled")
    assert rowptr.dtype == torch.int64 and col.dtype == torch.int32 and err.dtype == torch.int32
    N = rowptr.numel() - 1
    Xr, ldx = rows16(X)
    nat.check(
        nat.lib().lakde_mstep_tc_tiled(
            nat.dtype_code(X), N, X.size(1), X.size(0), nat.ptr(rowptr), nat.ptr(col), nat.ptr(order), nat.ptr(r),
            nat.ptr(Xr), ldx, int(kernel_offset), float(nu_0), nat.ptr(SP), nat.ptr(nu), nat.ptr(queue),
            nat.ptr(err), nat.stream_of(X),
        ),
        "mstep_tc_tiled",
    )


def posterior_factor_tiled(SP, D, jitter, eps, nu_0, a, b, out, logdet, info, T_tiles=None, trace=None,
                           X_tiles=None, W_cores=None):
    """posterior_factor from the tiled SP (and T) layout (see include/lakde_b200.h); writes W_triu to
    ``out``, X = W_triu^T as tiles to ``X_tiles`` and / or the W cores to ``W_cores``
    (any two may be None)."""
    nat.require_cuda(SP, jitter, nu_0, a, b, out, X_tiles, W_cores, logdet, info, T_tiles, trace,
                     op="posterior_factor_tiled")
    N = jitter.numel()
    if W_cores is not None:
        assert W_cores.dtype == torch.float32 and W_cores.is_contiguous()
        assert W_cores.numel() == N * int(nat.lib().lakde_w_cores_floats(int(D)))
    nat.check(
        nat.lib().lakde_posterior_factor_tiled(
            nat.dtype_code(SP), N, int(D), nat.ptr(SP), nat.ptr(nu_0), nat.ptr(a), nat.ptr(b), nat.ptr(jitter),
            float(eps), nat.ptr(out), nat.ptr(X_tiles), nat.ptr(W_cores), nat.ptr(logdet), nat.ptr(info),
            nat.ptr(T_tiles), nat.ptr(trace), nat.stream_of(SP),
        ),
        "posterior_factor_tiled",
    )


def weighted_gram(W_triu, w, out=None, workspace=None):
    """sum_n w_n W_triu_n W_triu_n^T in float64, [D, D] (see include/lakde_b200.h)."""
    nat.require_cuda(W_triu, w, out, op="weighted_gram")
    N, D, _ = W_triu.shape
    W_triu = W_triu.contiguous()
    w = w.to(W_triu.dtype).contiguous()
    out = torch.empty(D, D, dtype=torch.float64, device=W_triu.device) if out is None else out
    need = int(nat.lib().lakde_weighted_gram_workspace(D))
    if workspace is None or workspace.numel() < need:
        workspace = torch.empty(need, dtype=torch.uint8, device=W_triu.device)
    nat.check(nat.lib().lakde_weighted_gram(nat.dtype_code(W_triu), N, D, nat.ptr(W_triu), nat.ptr(w), nat.ptr(out),
                                            nat.ptr(workspace), workspace.numel(), nat.stream_of(W_triu)),
              "weighted_gram")
    return out


def knn_select(dist, X, row0, k, include_self=False, out_idx=None, out_dist=None):
    """The k nearest points of rows row0 .. row0 + nb - 1 from their float64
    squared distances dist [nb, N] to all rows of X [N, D] (float64), nearest
    first, ties by index, re-ranked by exact differences (lakde_knn_select,
    see include/lakde_b200.h).  out_idx [nb, k] int32 or int64 (int64 if not
    given); out_dist [nb, k] float32 or float64 (optional)."""
    nat.require_cuda(dist, X, out_idx, out_dist, op="knn_select")
    nb, N = dist.shape
    dist = dist.contiguous()
    X = X.contiguous()
    if dist.dtype != torch.float64 or X.dtype != torch.float64:
        raise TypeError("knn_select: dist and X must be float64")
    if out_idx is None:
        out_idx = torch.empty(nb, k, dtype=torch.int64, device=dist.device)
    dist_code = nat.dtype_code(out_dist) if out_dist is not None else 0
    nat.check(nat.lib().lakde_knn_select(nat.ptr(dist), nb, N, int(row0), nat.ptr(X), X.size(1), int(bool(include_self)),
                                         int(k), nat.dtype_code(out_idx), nat.ptr(out_idx), dist_code,
                                         nat.ptr(out_dist) if out_dist is not None else None, nat.stream_of(dist)),
              "knn_select")
    return out_idx


def knn_elbo(a, b, nu, logdet_W, logdet_sigma_0, mm, c, a_0, b_0, nu_0, D, out=None, workspace=None):
    """ELBO of LocalKNearestKDE in float64 as a 0-dim device tensor (see include/lakde_b200.h)."""
    nat.require_cuda(a, b, nu, logdet_W, logdet_sigma_0, mm, c, op="knn_elbo")
    dev = a.device
    out = torch.empty((), dtype=torch.float64, device=dev) if out is None else out
    need = nat.lib().lakde_knn_elbo_workspace()
    if workspace is None or workspace.numel() < need:
        workspace = torch.empty(need, dtype=torch.uint8, device=dev)
    nat.check(
        nat.lib().lakde_knn_elbo(
            nat.dtype_code(a), a.numel(), int(D), nat.ptr(a), nat.ptr(b), nat.ptr(nu), nat.ptr(logdet_W),
            nat.ptr(logdet_sigma_0), nat.ptr(mm), nat.ptr(c), float(a_0), float(b_0), float(nu_0),
            nat.ptr(workspace), workspace.numel(), nat.ptr(out), nat.stream_of(a),
        ),
        "knn_elbo",
    )
    return out


def knn_elbo_parts(D, a_0, b_0, nu_0, a=None, b=None, nu=None, logdet_W=None, logdet_sigma_0=None, mm=None, c=None,
                   tail=0.0, out=None, workspace=None, device=None):
    """float64 sum of the ELBO's kernel terms (a .. mm given) and / or point
    terms (c given) plus `tail`, as a 0-dim device tensor (see include/lakde_b200.h)."""
    nat.require_cuda(a, b, nu, logdet_W, logdet_sigma_0, mm, c, op="knn_elbo_parts")
    ref = a if a is not None else c
    dev = ref.device if ref is not None else device
    out = torch.empty((), dtype=torch.float64, device=dev) if out is None else out
    need = nat.lib().lakde_knn_elbo_workspace()
    if workspace is None or workspace.numel() < need:
        workspace = torch.empty(need, dtype=torch.uint8, device=dev)
    nk = 0 if a is None else a.numel()
    npts = 0 if c is None else c.numel()
    dtype = nat.dtype_code(ref) if ref is not None else nat.F32
    with torch.cuda.device(dev):
        nat.check(
            nat.lib().lakde_knn_elbo_parts(
                dtype, nk, npts, int(D), nat.ptr(a), nat.ptr(b), nat.ptr(nu), nat.ptr(logdet_W),
                nat.ptr(logdet_sigma_0), nat.ptr(mm), nat.ptr(c), float(a_0), float(b_0), float(nu_0), float(tail),
                nat.ptr(workspace), workspace.numel(), nat.ptr(out), nat.stream_of(out),
            ),
            "knn_elbo_parts",
        )
    return out


def log_pred_density_tc(X, W_cores, nu, log_coeff, Y, err, out=None, workspace=None):
    """log_pred_density with the quad forms on the tensor cores (tf32 hi / lo),
    float32, D <= 64, W_triu given as W cores (see include/lakde_b200.h)."""
    nat.require_cuda(X, W_cores, nu, log_coeff, Y, err, op="log_pred_density_tc")
    N, D = X.shape
    Nq = Y.size(0)
    out = Y.new_empty(Nq) if out is None else out
    if Nq == 0:
        return out
    Xr, ldx = rows16(X)
    Yr, ldy = rows16(Y.to(X.dtype))
    need = nat.lib().lakde_log_pred_density_tc_workspace(N, Nq, D)
    if workspace is None or workspace.numel() < need:
        workspace = torch.empty(need, dtype=torch.uint8, device=X.device)
    nat.check(
        nat.lib().lakde_log_pred_density_tc(
            nat.dtype_code(X), N, Nq, D, nat.ptr(Xr), ldx, nat.ptr(W_cores), nat.ptr(nu), nat.ptr(log_coeff),
            nat.ptr(Yr), ldy, nat.ptr(out), nat.ptr(workspace), workspace.numel(), nat.ptr(err), nat.stream_of(X),
        ),
        "log_pred_density_tc",
    )
    return out


def log_pred_density_bwd(X, W_triu, nu, log_coeff, Y, out, grad_out):
    """Pair pass of the predictive-density backward (see include/lakde_b200.h).

    Returns (grad_Y [Nq, D], sw [N], S_c [N, D, D]); the [N, Nq] weights are a
    temporary of the call.
    """
    nat.require_cuda(X, W_triu, nu, log_coeff, Y, out, grad_out, op="log_pred_density_bwd")
    N, D = X.shape
    Nq = Y.size(0)
    Y = Y.contiguous()
    grad_out = grad_out.contiguous()
    gY = torch.empty_like(Y)
    cw = X.new_empty(N, Nq)
    sw = X.new_empty(N)
    S_c = X.new_empty(N, D, D)
    need = int(nat.lib().lakde_log_pred_density_bwd_workspace(nat.dtype_code(X), N, Nq, D))
    ws = torch.empty(max(need, 1), dtype=torch.uint8, device=X.device)
    nat.check(
        nat.lib().lakde_log_pred_density_bwd(
            nat.dtype_code(X), N, Nq, D, nat.ptr(X), nat.ptr(W_triu), nat.ptr(nu), nat.ptr(log_coeff), nat.ptr(Y),
            nat.ptr(out), nat.ptr(grad_out), nat.ptr(gY), nat.ptr(cw), nat.ptr(sw), nat.ptr(S_c), nat.ptr(ws),
            ws.numel(), nat.stream_of(X),
        ),
        "log_pred_density_bwd",
    )
    return gY, sw, S_c


def estep_tc(rowptr, col, X, W_cores, nu, logdet_W, err, order=None, out=None, kernel_offset=0, queue=None):
    """Tensor-core (tf32 hi / lo) E-step numerators, D <= 64, W_triu given as W
    cores (see include/lakde_b200.h).  Row n of rowptr is kernel n + kernel_offset of X."""
    nat.require_cuda(rowptr, col, X, W_cores, nu, logdet_W, err, order, queue, op="estep_tc")
    assert rowptr.dtype == torch.int64 and col.dtype == torch.int32 and err.dtype == torch.int32
    assert W_cores.dtype == torch.float32 and W_cores.is_contiguous()
    N = rowptr.numel() - 1
    out = X.new_empty(col.numel()) if out is None else out
    Xr, ldx = rows16(X)
    nat.check(
        nat.lib().lakde_estep_tc(
            nat.dtype_code(X), N, X.size(1), X.size(0), nat.ptr(rowptr), nat.ptr(col), nat.ptr(order), nat.ptr(Xr),
            ldx, int(kernel_offset), nat.ptr(W_cores), nat.ptr(nu), nat.ptr(logdet_W), nat.ptr(out),
            nat.ptr(queue), nat.ptr(err), nat.stream_of(X),
        ),
        "estep_tc",
    )
    return out


def mstep_tc(rowptr, col, r, X, nu_0, err, order=None, S=None, nu=None, lower_only=False, kernel_offset=0,
             queue=None):
    """Tensor-core (tf32 hi / lo) M-step S and nu, D <= 64 (see include/lakde_b200.h).

    ``lower_only=True`` writes only the lower triangle of each S_n; row n of
    rowptr is kernel n + kernel_offset of X."""
    nat.require_cuda(rowptr, col, r, X, err, order, queue, op="mstep_tc")
    assert rowptr.dtype == torch.int64 and col.dtype == torch.int32 and err.dtype == torch.int32
    N = rowptr.numel() - 1
    D = X.size(1)
    S = X.new_empty(N, D, D) if S is None else S
    nu = X.new_empty(N) if nu is None else nu
    Xr, ldx = rows16(X)
    nat.check(
        nat.lib().lakde_mstep_tc(
            nat.dtype_code(X), N, D, X.size(0), nat.ptr(rowptr), nat.ptr(col), nat.ptr(order), nat.ptr(r),
            nat.ptr(Xr), ldx, int(kernel_offset), float(nu_0), nat.ptr(S), nat.ptr(nu), int(bool(lower_only)),
            nat.ptr(queue), nat.ptr(err), nat.stream_of(X),
        ),
        "mstep_tc",
    )
    return S, nu
