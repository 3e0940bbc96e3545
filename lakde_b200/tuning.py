"""Autotuner of the launch choices of the library.

Some kernels have more than one launch form that computes the same values
(``lakde_tuning_set`` in include/lakde_b200.h): the FP64 factorisation with two
warps per block or a lean form with one warp per block and 11 blocks per SM,
the tensor-core kernels with their rows from an atomic work queue or on a
static stride, the fused D <= 8 pass with a kernel row's pairs on two lanes
(its FP64 posterior on one lane per row) or with one thread per kernel row.  Which is faster depends on D, N and the pair counts, so the
fused engine times every choice on its own data before its first CUDA-graph
capture and keeps the fastest, per knob and class of D (the library's table
is process-wide).  The factorisation and row-schedule choices give identical
results; the two forms of the fused D <= 8 pass sum a row's pairs in
different orders, so they agree to rounding.  The state the timed launches
modify is saved and restored around the tuning.
"""

import torch

from . import _native as nat

# knob: (library index, choice names, the engine launches it affects)
KNOBS = {
    "factor": (0, ("two_warps_per_block", "one_warp_per_block_11_per_sm"), ("posterior_factor",)),
    "rows": (1, ("work_queue", "static_stride"), ("mstep_tc", "estep_tc")),
    "vi_rows": (2, ("two_lanes_per_row", "thread_per_row"), ("vi_rows",)),
}


def set_choice(knob, D, choice):
    idx, names, _ = KNOBS[knob]
    nat.check(nat.lib().lakde_tuning_set(idx, int(D), names.index(choice)), "tuning_set")


def get_choice(knob, D):
    idx, names, _ = KNOBS[knob]
    return names[nat.lib().lakde_tuning_get(idx, int(D))]


def _time(fns, reps):
    stream = torch.cuda.current_stream()
    for f in fns:  # warm-up (lazy allocations, instruction cache)
        f()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(reps):
        for f in fns:
            f()
    b.record(stream)
    torch.cuda.synchronize()
    return a.elapsed_time(b) / reps


def tune_engine(eng, reps=3):
    """Times each choice of each knob on the engine's launches (from
    ``eng.kernel_launches()``), sets the fastest and returns
    {knob: {"choice": name, "ms": {choice: ms per iteration}}}."""
    launches = eng.kernel_launches()
    snap = eng.snapshot()
    out = {}
    try:
        for knob, (_, names, affected) in KNOBS.items():
            fns = [launches[k] for k in affected if k in launches]
            if not fns:
                continue
            ms = {}
            for name in names:
                set_choice(knob, eng.D, name)
                ms[name] = round(_time(fns, reps), 4)
            best = min(ms, key=ms.get)
            set_choice(knob, eng.D, best)
            out[knob] = {"choice": best, "ms": ms}
    finally:
        eng.restore(snap)
    return out
