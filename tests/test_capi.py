"""The C-ABI library: it loads without a GPU, exports every entry point the
header declares, and rejects bad arguments before touching the device."""

import ctypes
import os
import re

import pytest
import torch

from .conftest import ROOT

HEADER = os.path.join(ROOT, "include", "lakde_b200.h")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"LAKDE_API\s+[\w\s\*]+?\b(lakde_\w+)\s*\(", text)))


@pytest.fixture(scope="module")
def nat():
    from lakde_b200 import _native

    return _native


def test_header_and_library_agree(nat):
    names = declared_symbols()
    assert len(names) >= 12
    lib = ctypes.CDLL(nat.library_path())
    for n in names:
        assert hasattr(lib, n), n
    assert sorted(nat.exported_symbols()) == names


def test_metadata(nat):
    lib = nat.lib()
    assert lib.lakde_abi_version() == 6
    assert lib.lakde_max_dim() == 64


def test_invalid_arguments_are_rejected_on_the_host(nat):
    lib = nat.lib()
    st = lib.lakde_W_inv(0, None, 2, None, 2, None, None, None, None, -1, 0, 3, None)
    assert st == 1
    assert b"invalid" in lib.lakde_last_error()
    assert lib.lakde_chol_quad_form(0, None, None, None, None, None, None, None, None, 1, 1, 0, None) == 1
    assert lib.lakde_ind2ptr(None, 2, 5, -1, None, 2, None) == 1
    assert lib.lakde_estep_normalise(0, 3, None, None, 2, None, None, None, None, 7, 0.0, None) == 1
    assert lib.lakde_log_pred_density_workspace(0, 100, 10, 65) == 0
    assert lib.lakde_log_pred_density_workspace(5, 100, 10, 8) == 0
    assert lib.lakde_log_pred_density_workspace(0, 100, 10, 8) > 0
    # an unsupported dtype code is reported as such
    assert lib.lakde_posterior_factor(7, 1, 2, ctypes.c_void_p(8), None, 0, None, None, None,
                                      ctypes.c_void_p(8), 0.0, ctypes.c_void_p(8), None, ctypes.c_void_p(8),
                                      ctypes.c_void_p(8), None, 0, 0, None, None, None) in (1, 2)
    # tensor-core entry points: rows of X must be 16-byte aligned (checked before any device work)
    p = ctypes.c_void_p(256)
    st = lib.lakde_estep_tc(0, 10, 63, 10, p, p, None, p, 63, 0, p, p, p, p, None, p, None)
    assert st == 1 and b"16-byte aligned rows" in lib.lakde_last_error()
    st = lib.lakde_mstep_tc(0, 10, 13, 10, p, p, None, p, ctypes.c_void_p(260), 16, 0, 14.0, p, p, 0, None, p, None)
    assert st == 1
    assert lib.lakde_estep_tc(1, 10, 8, 10, p, p, None, p, 8, 0, p, p, p, p, None, p, None) == 2
    assert lib.lakde_estep_tc(0, 10, 65, 10, p, p, None, p, 68, 0, p, p, p, p, None, p, None) == 4
    assert lib.lakde_w_cores_floats(63) == 36 * 128
    assert lib.lakde_w_cores_floats(21) == 6 * 128
    assert lib.lakde_w_cores_floats(3) == 128
    assert lib.lakde_w_cores_floats(65) == 0
    # kNN selection: sizes, k against the candidate count, dtypes and the
    # shared-memory bound of the candidate buffer, all before device work
    assert lib.lakde_knn_select(p, 4, 10, 0, p, 3, 0, 10, 2, p, 0, None, None) == 1
    assert b"exceeds" in lib.lakde_last_error()
    assert lib.lakde_knn_select(p, 4, 10, 8, p, 3, 0, 5, 2, p, 0, None, None) == 1
    assert lib.lakde_knn_select(p, 4, 10, 0, p, 3, 1, 10, 0, p, 0, None, None) == 1
    assert lib.lakde_knn_select(p, 4, 100000, 0, p, 3, 0, 20000, 3, p, 0, None, None) == 4
    assert b"shared memory" in lib.lakde_last_error()


def test_cpu_tensors_are_rejected():
    from lakde_b200 import kernels

    W = torch.eye(3).expand(4, 3, 3).contiguous()
    X = torch.zeros(4, 3)
    with pytest.raises((RuntimeError, NotImplementedError)):
        kernels.chol_quad_form(W, X, X)
    with pytest.raises((RuntimeError, NotImplementedError)):
        kernels.ind2ptr(torch.zeros(3, dtype=torch.int64), 4)
    with pytest.raises((RuntimeError, NotImplementedError)):
        kernels.calc_W_inv(torch.zeros(5, dtype=torch.int64), torch.zeros(0, dtype=torch.int64), torch.zeros(0),
                           X, X)


def test_tuning_table_round_trip_and_rejects_bad_choices(nat):
    """lakde_tuning_set / _get: one entry per knob and class of D (<= 16, 32,
    48, 64); unknown knobs, out-of-range D and choices are rejected."""
    from lakde_b200 import tuning

    lib = nat.lib()
    saved = {(k, d): lib.lakde_tuning_get(idx, d) for k, (idx, _, _) in tuning.KNOBS.items() for d in (8, 21, 40, 63)}
    try:
        for knob, (idx, names, _) in tuning.KNOBS.items():
            for d_set, d_same, d_other in ((8, 16, 17), (21, 32, 33), (40, 48, 49), (63, 64, 16)):
                for choice in names:
                    tuning.set_choice(knob, d_set, choice)
                    assert tuning.get_choice(knob, d_same) == choice
                other = names[0]
                tuning.set_choice(knob, d_set, other)
                tuning.set_choice(knob, d_other, names[1])
                assert tuning.get_choice(knob, d_set) == other
        assert lib.lakde_tuning_set(3, 8, 0) != 0
        assert lib.lakde_tuning_set(-1, 8, 0) != 0
        assert lib.lakde_tuning_set(0, 0, 0) != 0
        assert lib.lakde_tuning_set(0, 65, 0) != 0
        assert lib.lakde_tuning_set(0, 8, 2) != 0
        assert "no choice" in lib.lakde_last_error().decode()
    finally:
        for (k, d), v in saved.items():
            assert lib.lakde_tuning_set(tuning.KNOBS[k][0], d, v) == 0
