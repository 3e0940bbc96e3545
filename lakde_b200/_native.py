"""ctypes binding of the CUDA library ``_lib/liblakde_b200.so`` (C ABI in
``include/lakde_b200.h``).

The library is the only compute path of this package: there is no CPU or
pure-PyTorch fallback.  If it is missing the first op call raises, naming the
build command.
"""

import ctypes
import os

import torch

from . import build as _build

F32, F64, I32, I64 = 0, 1, 2, 3
_DTYPE_CODES = {torch.float32: F32, torch.float64: F64, torch.int32: I32, torch.int64: I64}

_c_i64 = ctypes.c_int64
_c_int = ctypes.c_int
_c_vp = ctypes.c_void_p
_c_dbl = ctypes.c_double

_SIGNATURES = {
    "lakde_last_error": ([], ctypes.c_char_p),
    "lakde_abi_version": ([], _c_int),
    "lakde_max_dim": ([], _c_int),
    "lakde_tuning_set": ([_c_int, _c_i64, _c_int], _c_int),
    "lakde_tuning_get": ([_c_int, _c_i64], _c_int),
    "lakde_ind2ptr": ([_c_vp, _c_int, _c_i64, _c_i64, _c_vp, _c_int, _c_vp], _c_int),
    "lakde_chol_quad_form": (
        [_c_int, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp, _c_i64, _c_i64, _c_i64, _c_vp],
        _c_int,
    ),
    "lakde_W_inv": (
        [_c_int, _c_vp, _c_int, _c_vp, _c_int, _c_vp, _c_vp, _c_vp, _c_vp, _c_i64, _c_i64, _c_i64, _c_vp],
        _c_int,
    ),
    "lakde_mstep": (
        [_c_int, _c_i64, _c_i64, _c_i64, _c_vp, _c_int, _c_vp, _c_int, _c_vp, _c_vp, _c_i64, _c_dbl, _c_vp, _c_vp,
         _c_vp],
        _c_int,
    ),
    "lakde_posterior_factor": (
        [_c_int, _c_i64, _c_i64, _c_vp, _c_vp, _c_i64, _c_vp, _c_vp, _c_vp, _c_vp, _c_dbl, _c_vp, _c_vp,
         _c_vp, _c_vp, _c_vp, _c_i64, _c_int, _c_vp, _c_vp, _c_vp],
        _c_int,
    ),
    "lakde_estep_logrho": (
        [_c_int, _c_i64, _c_i64, _c_i64, _c_vp, _c_int, _c_vp, _c_int, _c_vp, _c_i64, _c_vp, _c_vp, _c_vp,
         _c_vp, _c_vp],
        _c_int,
    ),
    "lakde_vi_rows": (
        [_c_int, _c_i64, _c_i64, _c_i64, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp, _c_i64, _c_dbl, _c_vp, _c_i64, _c_vp, _c_i64,
         _c_vp, _c_vp, _c_dbl, _c_vp, _c_dbl, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp],
        _c_int,
    ),
    "lakde_estep_tc": (
        [_c_int, _c_i64, _c_i64, _c_i64, _c_vp, _c_vp, _c_vp, _c_vp, _c_i64, _c_i64, _c_vp, _c_vp, _c_vp, _c_vp,
         _c_vp, _c_vp, _c_vp],
        _c_int,
    ),
    "lakde_mstep_tc": (
        [_c_int, _c_i64, _c_i64, _c_i64, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp, _c_i64, _c_i64, _c_dbl, _c_vp, _c_vp,
         _c_int, _c_vp, _c_vp, _c_vp],
        _c_int,
    ),
    "lakde_w_cores_floats": ([_c_i64], ctypes.c_size_t),
    "lakde_tc_wait_timeout_probe": (
        [_c_i64, _c_i64, _c_i64, _c_vp, _c_vp, _c_vp, _c_i64, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp],
        _c_int,
    ),
    "lakde_pack_w_cores": ([_c_int, _c_i64, _c_i64, _c_vp, _c_vp, _c_vp], _c_int),
    "lakde_estep_normalise": (
        [_c_int, _c_i64, _c_vp, _c_vp, _c_int, _c_vp, _c_vp, _c_vp, _c_vp, _c_int, _c_dbl, _c_vp],
        _c_int,
    ),
    "lakde_estep_normalise_stage": (
        [_c_int, _c_int, _c_i64, _c_vp, _c_vp, _c_int, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp, _c_int, _c_dbl,
         _c_vp],
        _c_int,
    ),
    "lakde_pred_coeff": ([_c_int, _c_i64, _c_i64, _c_vp, _c_vp, _c_vp, _c_vp], _c_int),
    "lakde_log_pred_density_workspace": ([_c_int, _c_i64, _c_i64, _c_i64], ctypes.c_size_t),
    "lakde_log_pred_density_bwd_workspace": ([_c_int, _c_i64, _c_i64, _c_i64], ctypes.c_size_t),
    "lakde_log_pred_density_bwd": (
        [_c_int, _c_i64, _c_i64, _c_i64, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp,
         _c_vp, _c_vp, ctypes.c_size_t, _c_vp],
        _c_int,
    ),
    "lakde_log_pred_density_noalloc": (
        [_c_int, _c_i64, _c_i64, _c_i64, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp],
        _c_int,
    ),
    "lakde_log_pred_density": (
        [_c_int, _c_i64, _c_i64, _c_i64, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp, ctypes.c_size_t, _c_vp],
        _c_int,
    ),
    "lakde_log_pred_density_tc_workspace": ([_c_i64, _c_i64, _c_i64], ctypes.c_size_t),
    "lakde_knn_elbo_workspace": ([], ctypes.c_size_t),
    "lakde_weighted_gram_workspace": ([_c_i64], ctypes.c_size_t),
    "lakde_weighted_gram": ([_c_int, _c_i64, _c_i64, _c_vp, _c_vp, _c_vp, _c_vp, ctypes.c_size_t, _c_vp], _c_int),
    "lakde_knn_select": (
        [_c_vp, _c_i64, _c_i64, _c_i64, _c_vp, _c_i64, _c_int, _c_i64, _c_int, _c_vp, _c_int, _c_vp, _c_vp],
        _c_int,
    ),
    "lakde_tile_count": ([_c_i64], _c_i64),
    "lakde_pack_tiles": ([_c_int, _c_i64, _c_i64, _c_vp, _c_i64, _c_vp, _c_i64, _c_i64, _c_i64, _c_vp], _c_int),
    "lakde_mstep_tc_tiled": (
        [_c_int, _c_i64, _c_i64, _c_i64, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp, _c_i64, _c_i64, _c_dbl, _c_vp, _c_vp,
         _c_vp, _c_vp, _c_vp],
        _c_int,
    ),
    "lakde_posterior_factor_tiled": (
        [_c_int, _c_i64, _c_i64, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp, _c_dbl, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp,
         _c_vp, _c_vp, _c_vp],
        _c_int,
    ),
    "lakde_knn_elbo": (
        [_c_int, _c_i64, _c_i64, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp, _c_dbl, _c_dbl, _c_dbl, _c_vp,
         ctypes.c_size_t, _c_vp, _c_vp],
        _c_int,
    ),
    "lakde_knn_elbo_parts": (
        [_c_int, _c_i64, _c_i64, _c_i64, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp, _c_dbl, _c_dbl, _c_dbl,
         _c_dbl, _c_vp, ctypes.c_size_t, _c_vp, _c_vp],
        _c_int,
    ),
    "lakde_log_pred_density_tc": (
        [_c_int, _c_i64, _c_i64, _c_i64, _c_vp, _c_i64, _c_vp, _c_vp, _c_vp, _c_vp, _c_i64, _c_vp, _c_vp,
         ctypes.c_size_t, _c_vp, _c_vp],
        _c_int,
    ),
}

_lib = None


def library_path():
    return _build.lib_path()


def lib():
    """The loaded library (loaded on first use)."""
    global _lib
    if _lib is None:
        path = library_path()
        if not os.path.exists(path):
            raise RuntimeError(
                f"lakde_b200 CUDA library not found at {path}; build it with "
                "`python -m lakde_b200.build` (there is no CPU fallback)"
            )
        handle = ctypes.CDLL(path)
        for name, (args, res) in _SIGNATURES.items():
            fn = getattr(handle, name)
            fn.argtypes = args
            fn.restype = res
        _lib = handle
    return _lib


def exported_symbols():
    return list(_SIGNATURES)


def check(status, what):
    if status != 0:
        msg = lib().lakde_last_error().decode(errors="replace")
        raise RuntimeError(f"lakde_b200 {what} failed (status {status}): {msg}")


def dtype_code(t):
    try:
        return _DTYPE_CODES[t.dtype]
    except KeyError:
        raise TypeError(f"unsupported dtype {t.dtype}") from None


def ptr(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def stream_of(t):
    return ctypes.c_void_p(torch.cuda.current_stream(t.device).cuda_stream)


def require_cuda(*tensors, op="op"):
    for t in tensors:
        if t is not None and not t.is_cuda:
            raise RuntimeError(
                f"lakde_b200 {op}: expected CUDA tensors (the kernels run on the GPU only), got {t.device}"
            )


def strides(t):
    return (ctypes.c_int64 * t.dim())(*t.stride())
