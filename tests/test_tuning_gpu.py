"""Every launch form the autotuner can pick computes the same iteration: the
FP64 factorisation with two warps per block or the lean one-warp form (its
trace tiles read from global memory), the tensor-core rows from the atomic
work queue or on a static stride (bit for bit), and the two forms of the
fused D <= 8 pass (to rounding: they sum a row's pairs in different orders).
Then the tuner itself: it times every choice and keeps the fastest."""

import numpy as np
import pytest
import torch

from oracle import lakde_oracle as O

pytestmark = pytest.mark.gpu
DEV = "cuda"

OUTPUTS = ("Wc", "trace", "logdet_W", "info", "W_inv_jitter", "SP", "S", "nu", "logrho", "b",
           "sigma_0_lambda_mm_trace")


@pytest.fixture
def table():
    from lakde_b200 import tuning

    saved = {(k, d): tuning.get_choice(k, d) for k in tuning.KNOBS for d in (8, 21, 40, 63)}
    yield tuning
    for (k, d), c in saved.items():
        tuning.set_choice(k, d, c)


def engine(D, precision, N=3000, k=24, seed=0):
    from lakde_b200.engine import FusedKNN
    from lakde_b200.sparse_util import PairPattern
    from lakde_b200.synthetic import wide_spectrum_mixture

    Xn, _ = wide_spectrum_mixture(seed=seed, n_train=N, n_test=1, d=D)
    X = torch.tensor(Xn, device=DEV)
    graph = torch.tensor(O.knn_graph(Xn.astype(np.float64), k).astype(np.int32), device=DEV)
    tiny = torch.tensor(1e-6, device=DEV)
    eng = FusedKNN(X, graph, PairPattern.from_knn_graph(graph), float(D), tiny, tiny, 5e-4, k, precision=precision)
    eng.init_summaries()
    eng.step()
    torch.cuda.synchronize()
    return eng


def outputs_per_choice(eng, tuning, knob):
    _, names, affected = tuning.KNOBS[knob]
    launches = eng.kernel_launches()
    fns = [launches[a] for a in affected if a in launches]
    assert fns, (knob, list(launches))
    snap = eng.snapshot()
    res = {}
    for name in names:
        eng.restore(snap)
        tuning.set_choice(knob, eng.D, name)
        for f in fns:
            f()
        torch.cuda.synchronize()
        res[name] = {k: getattr(eng, k).clone() for k in OUTPUTS if torch.is_tensor(getattr(eng, k, None))}
    eng.restore(snap)
    eng.check_errors()
    return res


@pytest.mark.parametrize("D", [21, 63])
@pytest.mark.parametrize("knob", ["factor", "rows"])
def test_tensor_core_path_launch_forms_agree_bit_for_bit(table, knob, D):
    eng = engine(D, "mixed")
    a, b = outputs_per_choice(eng, table, knob).values()
    for k in a:
        torch.testing.assert_close(a[k], b[k], rtol=0, atol=0, equal_nan=True, msg=f"{knob} {k}")


@pytest.mark.parametrize("D", [3, 8])
def test_fused_row_pass_forms_agree_to_rounding(table, D):
    eng = engine(D, "fp32")
    a, b = outputs_per_choice(eng, table, "vi_rows").values()
    # log rho = c0 - nu / 2 Q of terms near 1e2 that partly cancel: rounding
    # differences of the two summation orders reach 1e-4 absolute there
    for k, (rtol, atol) in (("logrho", (1e-4, 1e-3)), ("nu", (1e-6, 0)), ("logdet_W", (1e-5, 1e-4)),
                            ("b", (1e-5, 0))):
        if k in a:
            torch.testing.assert_close(a[k], b[k], rtol=rtol, atol=atol, equal_nan=True)


def test_tuner_times_every_choice_and_keeps_the_fastest(table):
    from lakde_b200.tuning import tune_engine

    eng = engine(21, "mixed")
    snap = eng.snapshot()
    out = tune_engine(eng, reps=2)
    assert set(out) == {"factor", "rows"}
    for knob, rec in out.items():
        names = table.KNOBS[knob][1]
        assert set(rec["ms"]) == set(names)
        assert rec["choice"] == min(rec["ms"], key=rec["ms"].get)
        assert table.get_choice(knob, 21) == rec["choice"]
    for k, v in snap.items():  # the state is restored after the timing
        torch.testing.assert_close(getattr(eng, k), v, rtol=0, atol=0, equal_nan=True)
