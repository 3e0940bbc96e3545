"""Benchmark of the lakde VI hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload bsds63|gas8|...]
                    [--impl reference] [--no-fp64-check] [--no-cpu-baseline]

A step is one VI iteration of LocalKNearestKDE over all N kernels (fused
batch schedule on the kNN candidate pattern), on seeded synthetic data with
the shape of the named workload; the default is the d=63, N=1,000,000, K=100
decaying-spectrum mixture in mixed precision (tensor-core tf32 hi / lo
contractions, FP64 factorisations).  Inputs are resident in HBM; L2 is
flushed between timed steps.  Rank 0 prints one JSON line with the whole-job
throughput, the roofline of the dominant kernel, the plain-FP32 arm timed
from the same state, the held-out log density of mixed precision, plain FP32
and FP64 after the same iterations from the same initialisation, the
end-to-end number through the public API with host buffers, the CPU baseline
(the same sparse schedule restated in numpy, timed on a bounded sample on all
host cores) and the SM clocks sampled during the timed region.
Under torchrun (N > 1), or with --sharded, the kernels are sharded over the
ranks (lakde_b200.shard: one VI iteration of the whole data set per step, the
per-point normaliser all-reduced over NCCL), so N GPUs share one problem
(strong scaling).
"""

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "VI iters/s and log_pred_density pts/s, mixed vs plain FP32 GPU at ≤1e-3 nats"

WORKLOADS = {
    # name: (generator kwargs, K, threshold, description)
    "gas8": (dict(n_train=200_000, n_test=20_000), 50, 5e-4,
             "LocalKNearestKDE d=8 N_train=200000 N_test=20000 K=50 (10-component heavy-tail mixture)"),
    "bsds63": (dict(n_train=1_000_000, n_test=16_384), 100, 5e-4,
               "LocalKNearestKDE d=63 N_train=1000000 N_test=16384 K=100 (20-component decaying-spectrum mixture)"),
    "bsds63s": (dict(n_train=50_000, n_test=2_048), 100, 5e-4,
                "LocalKNearestKDE d=63 N_train=50000 N_test=1024 K=100 (the bsds63 mixture, small case for "
                "profiling)"),
    "spec21": (dict(n_train=300_000, n_test=4_096), 64, 5e-4,
               "LocalKNearestKDE d=21 N_train=300000 N_test=4096 K=64 (12-component mixture)"),
    "circle2d": (dict(n_train=2_000, n_test=1_000), 20, 0.0,
                 "LocalKNearestKDE d=2 N_train=2000 N_test=1000 K=20 (8-Gaussian circle)"),
    # hierarchical model (run_hier): K is the kNN seed of the responsibilities
    "embed43": (dict(n_train=30_000, n_test=3_000), 16, 0.0,
                "LocalHierarchicalKDE d=43 N_train=30000 N_test=3000 (10-dim 6-component mixture embedded in 43 "
                "dims, noise sd 1e-3), lognormal neighbourhoods median 64 sigma 1 cap 4096"),
}


def make_data(name):
    from lakde_b200 import synthetic as syn

    kw, k, thr, desc = WORKLOADS[name]
    gen = {"gas8": syn.heavy_tail_mixture, "bsds63": syn.decaying_spectrum_mixture,
           "bsds63s": syn.decaying_spectrum_mixture, "embed43": syn.embedded_mixture,
           "spec21": syn.wide_spectrum_mixture, "circle2d": syn.circle_gmm}[name]
    Xtr, Xte = gen(seed=0, **kw)
    return Xtr, Xte, k, thr, desc


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def load_traffic(kernel, workload):
    """Per-launch DRAM bytes of `kernel` from a committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        d = json.load(f)
    v = d.get(workload, {}).get(kernel)
    return None if v is None else float(v)


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons while the timed region runs."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.samples = []
        self.proc = None
        self.thread = None

    def wait_for_samples(self, n, timeout_s, keep_busy):
        """Keeps the GPU busy until the sampler has produced n samples."""
        t0 = time.perf_counter()
        while len(self.samples) < n and time.perf_counter() - t0 < timeout_s:
            keep_busy()

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 8:
                self.samples.append(parts)

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        return False

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for s in self.samples for n, v in zip(names, s[4:8]) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def alg_flops(N, D, nnz):
    """Algorithmic flops per launch: nnz 2T for the triangular quad forms and for
    the rank-one scatter (T = D (D + 1) / 2), D^3 / 3 each for the FP64 Cholesky,
    inverse and trace products."""
    T = D * (D + 1) // 2
    return {"mstep": 2 * T * nnz, "mstep_tc": 2 * T * nnz, "estep_logrho": 2 * T * nnz, "estep_tc": 2 * T * nnz,
            "posterior_factor": N * D ** 3}


def alg_bytes(N, D, nnz, es=4):
    """Compulsory bytes per launch of the kernels of one iteration (each array
    once; triangular matrices count their triangle, T = D (D + 1) / 2)."""
    T = D * (D + 1) // 2
    b = {
        # rowptr, order, col, r, X, prior P and factor L0, per-kernel vectors, logrho
        "vi_rows": 8 * (N + 1) + 4 * N + 4 * nnz + es * nnz + es * N * D + 2 * es * N * T + 8 * es * N + es * nnz,
        # rowptr, col, r, X; S (symmetric: its triangle) and nu out
        "mstep": 8 * (N + 1) + 4 * nnz + es * nnz + es * N * D + es * N * T + es * N,
        # S, P, L0 in, W_triu out (triangles); nu, a, b, jitter in; logdet, trace, jitter, info out
        "posterior_factor": 4 * es * N * T + 4 * es * N + 3 * es * N + 4 * N,
        # rowptr, col, X, W_triu (triangle), nu, logdet in; logrho out
        "estep_logrho": 8 * (N + 1) + 4 * nnz + es * N * D + es * N * T + 2 * es * N + es * nnz,
        "estep_normalise": 8 * (N + 1) + 4 * nnz + es * nnz + es * nnz + 4 * es * N,
    }
    b["mstep_tc"] = b["mstep"]
    b["estep_tc"] = b["estep_logrho"]
    return b


def timed_steps(eng, steps, flush, torch):
    """Times each VI iteration (the product step) with CUDA events, L2 flushed before each."""
    stream = torch.cuda.current_stream()
    total = 0.0
    for _ in range(steps):
        flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        eng.step()
        b.record(stream)
        torch.cuda.synchronize()
        total += a.elapsed_time(b)
    return total


def kernel_split(eng, reps, flush, torch):
    """Average duration of each library kernel of the iteration, timed one by one."""
    stream = torch.cuda.current_stream()
    launches = eng.kernel_launches()
    out = {k: 0.0 for k in launches}
    for _ in range(reps):
        for name, fn in launches.items():
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            torch.cuda.synchronize()
            out[name] += a.elapsed_time(b)
    return {k: v / reps for k, v in out.items()}


def _cpu_rows(job):
    """One chunk of kernel rows of a VI iteration on the kNN pattern, in the
    oracle's numpy restatement of the reference arithmetic: M-step (scatter
    covariance and nu), jittered FP64 Cholesky, triangular inverse, log det and
    trace, then the E-step numerators of the rows' pairs.  Returns the seconds
    it took (run in a spawned worker process)."""
    import time as _time

    from oracle import lakde_oracle as O

    Xs, rowptr, col, r, self_idx, sigma0, L0, nu0, scale = job
    t0 = _time.perf_counter()
    Xn = Xs[self_idx]
    S = O.calc_W_inv(rowptr, col, r, Xn, Xs)
    rows = O._rows_of(rowptr)
    # per-row sums of r (rows without pairs, last in the longest-first order, sum to 0)
    nu = nu0 + np.bincount(rows, weights=r, minlength=len(self_idx))
    A = (sigma0 * scale[:, None, None] + S).astype(np.float64)
    L, _ = O.stabilized_cholesky(A, eps=float(np.finfo(np.float32).eps))
    W = np.swapaxes(O.tril_inverse(L), -1, -2)
    logdet = O.chol_logdet(W)
    O.chol_mm_trace(L0.astype(np.float64), W)
    delta = Xs[col] - Xn[rows]
    y = np.einsum("pji,pj->pi", np.triu(W)[rows], delta, optimize=True)
    Q = (y * y).sum(-1)
    _ = Q * (-0.5 * nu[rows]) + O.log_rho_const(nu, logdet, Xs.shape[1])[rows]
    return _time.perf_counter() - t0


def cpu_baseline(Xtr, rows_source, sigma0_fn, n_rows, nnz, k, thr, nu0, budget_s=20.0, procs=None,
                 order_note="in the GPU's longest-first order"):
    """The same sparse schedule as the GPU step, restated in numpy (the oracle),
    timed on a bounded sample on the host cores.  rows_source(start, count)
    gives kernel rows in the GPU's visiting order (longest first) as (rows,
    CSR pointer, pair points); chunks of rows go to a pool of spawned worker
    processes, one chunk each, until the budget is spent, and the normaliser
    pass is timed on as many pairs.  One VI iteration = the per-row time scaled
    to all n_rows rows plus the normaliser scaled to all nnz pairs."""
    import multiprocessing as mp

    from oracle import lakde_oracle as O

    D = Xtr.shape[1]
    procs = procs or os.cpu_count() or 1
    ctx = mp.get_context("spawn")
    rows_per_job = 64 if D > 32 else 256
    done_rows = done_pairs = 0
    wall = 0.0
    rng = np.random.default_rng(0)
    with ctx.Pool(procs) as pool:
        start = 0
        while wall < budget_s and start < n_rows:
            jobs = []
            for _ in range(procs):
                rows, sub_ptr, pts = rows_source(start, rows_per_job)
                start += rows_per_job
                if len(rows) == 0:
                    break
                uniq, inv = np.unique(np.concatenate([rows, pts]), return_inverse=True)
                Xs = Xtr[uniq].astype(np.float32)
                sig0, L0 = sigma0_fn(rows)
                r = rng.uniform(0.0, 2.0 / k, len(pts)).astype(np.float32)
                scale = np.full(len(rows), nu0, np.float32)
                jobs.append((Xs, sub_ptr, inv[len(rows):], r, inv[:len(rows)], sig0, L0, nu0, scale))
                done_rows += len(rows)
                done_pairs += len(pts)
            if not jobs:
                break
            t0 = time.perf_counter()
            pool.map(_cpu_rows, jobs)
            wall += time.perf_counter() - t0
    # the normaliser over as many pairs as the sample had (scatter / gather passes)
    m = max(1, min(done_pairs, nnz))
    npt = max(1, m // k)
    colm = rng.integers(0, npt, m)
    lr = rng.normal(-5, 3, m).astype(np.float32)
    t0 = time.perf_counter()
    O.sparse_normalise(colm, lr, np.zeros(npt, np.float32), np.ones(npt, np.float32), npt, 1, thr)
    t_norm = time.perf_counter() - t0
    per_iter = wall * n_rows / max(done_rows, 1) + t_norm * nnz / m
    return {
        "value": 1.0 / per_iter,
        "unit": "VI iters/s",
        "cores": procs,
        "kind": "port",
        "sample": (f"the GPU step's sparse schedule (kNN pattern, block = N) in the oracle's numpy restatement: "
                   f"{done_rows} of {n_rows} kernel rows {order_note} ({done_pairs} pairs: "
                   f"M-step, FP64 jittered Cholesky, inverse, trace, E-step numerators) in {wall:.1f} s on {procs} "
                   f"spawned processes, plus the normaliser on {m} pairs ({t_norm:.2f} s); scaled to {n_rows} "
                   f"rows and {nnz} pairs"),
    }


def pattern_rows_source(rowptr, col, order):
    """rows_source of cpu_baseline over a host copy of the engine's pattern."""
    def source(start, count):
        rows = order[start:start + count].astype(np.int64)
        lo, hi = rowptr[rows], rowptr[rows + 1]
        ptr = np.concatenate([[0], np.cumsum(hi - lo)]).astype(np.int64)
        pts = np.concatenate([col[a:b] for a, b in zip(lo, hi)]) if len(rows) else np.zeros(0, np.int64)
        return rows, ptr, pts.astype(np.int64)
    return source


def run_reference(args):
    """The reference arm: the CPU restatement of the same sparse schedule timed
    on the host cores (rank 0 only); each step is one bounded sample.  Kernel
    rows of the sample take the k nearest neighbours of their centre among a
    pool of 50,000 points as their pairs (the pattern's rows hold k pairs on
    average), and a kNN covariance of the same pool as their prior."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    Xtr, Xte, k, thr, desc = make_data(args.workload)
    N, D = Xtr.shape
    rng = np.random.default_rng(0)
    perm = rng.permutation(N)
    pool = Xtr[: min(N, 50_000)].astype(np.float64)
    pool_sq = (pool * pool).sum(1)
    nbr_cache = {}

    def knn_rows(rows):
        # squared distances by |x|^2 + |p|^2 - 2 x.p (one GEMM, no [rows, pool, D] temporary)
        key = (int(rows[0]), len(rows)) if len(rows) else None
        if key not in nbr_cache:
            xr = Xtr[rows].astype(np.float64)
            d = (xr * xr).sum(1)[:, None] + pool_sq[None, :] - 2.0 * (xr @ pool.T)
            nbr_cache.clear()
            nbr_cache[key] = np.argpartition(d, k, axis=1)[:, :k]
        return nbr_cache[key]

    def source(start, count):
        rows = perm[start:start + count].astype(np.int64)
        nbr = knn_rows(rows)
        ptr = np.arange(0, (len(rows) + 1) * k, k, dtype=np.int64)
        return rows, ptr, nbr.reshape(-1).astype(np.int64)

    def sigma0_fn(rows):
        nbr = knn_rows(rows)
        diff = pool[nbr] - Xtr[rows][:, None, :]
        sig = np.einsum("nki,nkj->nij", diff, diff) / k + 1e-6 * np.eye(D)
        return sig.astype(np.float32), np.linalg.cholesky(sig).astype(np.float32)

    vals = []
    t0 = time.perf_counter()
    for _ in range(max(1, args.steps)):
        vals.append(cpu_baseline(Xtr, source, sigma0_fn, N, N * k, k, thr, float(D), budget_s=8.0,
                                 order_note="in random order, each with its k nearest neighbours as pairs"))
        if time.perf_counter() - t0 > 100.0:
            break
    v = statistics.median([x["value"] for x in vals])
    cb = dict(vals[-1])
    cb["value"] = v
    args.steps = len(vals)
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "VI iters/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"{args.workload}: {desc}",
                   "schedule": "fused batch VI (block_size=N) on the kNN candidate pattern, numpy restatement"},
        "cpu_baseline": cb,
        "e2e": {"value": v, "unit": "VI iters/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def _block_knn(X, k, rows):
    X64 = X.astype(np.float64)
    out = np.empty((rows, k), dtype=np.int64)
    for s in range(0, rows, 256):
        d = ((X64[s:s + 256, None, :] - X64[None]) ** 2).sum(-1)
        d[np.arange(min(256, rows - s)), s + np.arange(min(256, rows - s))] = np.inf
        part = np.argpartition(d, k, axis=1)[:, :k]
        dd = np.take_along_axis(d, part, 1)
        out[s:s + 256] = np.take_along_axis(part, np.argsort(dd, axis=1, kind="stable"), 1)
    return out


def fp64_check(Xtr, Xte, graph, thr, iters, dev):
    """Held-out mean log density and ELBO after `iters` VI iterations from the
    same initialisation (same data, kNN graph and pattern) in mixed precision,
    plain FP32 and FP64; each model is freed before the next is built."""
    import torch

    from lakde_b200 import LocalKNearestKDE

    out = {"iterations": iters, "queries": int(len(Xte))}
    for name, dt, prec in (("mixed", torch.float32, "mixed"), ("plain_fp32", torch.float32, "fp32"),
                           ("fp64", torch.float64, "fp32")):
        X = torch.tensor(Xtr, dtype=dt, device=dev)
        Y = torch.tensor(Xte, dtype=dt, device=dev)
        m = LocalKNearestKDE(k_or_knn_graph=graph, fused=True, cuda_graph=True, precision=prec)
        m.fit(X, iterations=iters, sparsity_threshold=thr)
        ll = m.log_pred_density(X, Y).double()
        out[name] = {"mean_log_density": float(ll.mean()), "elbo": float(m.compute_elbo(X))}
        m.check_errors_()
        del m, X, Y, ll
        torch.cuda.empty_cache()
    ref = out["fp64"]["mean_log_density"]
    out["mixed_vs_fp64_nats"] = abs(out["mixed"]["mean_log_density"] - ref)
    out["plain_fp32_vs_fp64_nats"] = abs(out["plain_fp32"]["mean_log_density"] - ref)
    return out


def run_sharded(args, world, rank, dev):
    """One VI iteration of the whole workload per step, kernels sharded over
    the ranks (strong scaling); timed as the max over ranks."""
    import torch
    import torch.distributed as dist

    from lakde_b200 import kernels as K
    from lakde_b200.shard import LocalComm, ShardedKNN, TorchComm
    from lakde_b200.sparse_util import PairPattern
    from lakde_b200.utils import compute_knn_graph

    Xtr, Xte, k, thr, desc = make_data(args.workload)
    X = torch.tensor(Xtr, device=dev)
    Y = torch.tensor(Xte, device=dev)
    N, D = X.shape
    comm = TorchComm() if world > 1 else LocalComm()
    t_init = time.perf_counter()
    graph = compute_knn_graph(X, k, 1024, include_self=False, metric="l2", dtype=torch.int32)
    pattern = PairPattern.from_knn_graph(graph)
    init_k = min(math.floor(1 / thr), k) if thr else k
    nu_0 = float(D)
    eng = ShardedKNN(X, graph, pattern, nu_0, 1e-6, 1e-6, thr, init_k, comm=comm, precision=args.precision)
    eng.init_summaries()
    torch.cuda.synchronize()
    t_init = time.perf_counter() - t_init
    for _ in range(args.warmup):
        eng.step()
    torch.cuda.synchronize()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def barrier():
        if world > 1:
            dist.barrier()

    def timed(fn, reps):
        tot = 0.0
        for _ in range(reps):
            flush.zero_()
            barrier()
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            fn()
            b.record()
            torch.cuda.synchronize()
            barrier()
            tot += a.elapsed_time(b)
        return tot / reps

    clocks = ClockSampler(dev.index).__enter__()

    def busy():
        for _ in range(10):
            eng.step()
        torch.cuda.synchronize()

    clocks.wait_for_samples(3, 20.0, busy)
    n_before = len(clocks.samples)
    ms = timed(eng.step, args.steps)
    clocks.wait_for_samples(n_before + 2, 20.0, busy)
    clocks.__exit__(None, None, None)
    # phase split on this rank (the normaliser includes its all-reduces)
    reps = max(3, args.steps // 2)
    if D <= 8:
        # the fused per-row pass of the shard (what eng.step runs for D <= 8)
        split = {
            "vi_rows": timed(
                lambda: eng.ops.vi_rows(eng.pat, eng.r, eng.X, eng.lo, eng.nu_0, eng.a, eng.b, eng.b_0,
                                        eng.W_inv_jitter, eng.eps, eng.nu, eng.logdet_W, eng.info, eng.logrho,
                                        eng.sigma_0, eng.sigma_0_tril, eng.mm), reps),
            "estep_normalise_stages+allreduce": timed(lambda: eng._normalise(1), reps),
        }
    else:
        split = {
            ("mstep_tc" if eng.precision == "mixed" else "mstep"): timed(eng._mstep, reps),
            "posterior_factor": timed(eng._factor, reps),
            ("estep_tc" if eng.precision == "mixed" else "estep_logrho"): timed(
                lambda: eng.ops.estep(eng.pat, eng.X, eng.lo, eng.U, eng.nu, eng.logdet_W, eng.logrho,
                                      eng.precision, eng.err, **eng._tc_kw(W_cores=eng.Wc)), reps),
            "estep_normalise_stages+allreduce": timed(lambda: eng._normalise(1), reps),
        }
    t = torch.tensor([ms], device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms = float(t)
    # end to end: host X copied into the engine's point buffer, one iteration,
    # the ELBO read back
    Xh = torch.tensor(Xtr).pin_memory()

    def e2e_step():
        eng.X.copy_(Xh, non_blocking=True)
        eng.step()
        return float(eng.compute_elbo())

    e2e_ms = timed(e2e_step, args.steps)
    t = torch.tensor([e2e_ms], device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    e2e_ms = float(t)
    elbo = float(eng.compute_elbo())
    lpd_ms = timed(lambda: eng.log_pred_density(Y), 2)
    lpd = eng.log_pred_density(Y)
    eng.check_errors()
    dom = max((k_ for k_ in split if k_ != "estep_normalise_stages+allreduce"), key=split.get)
    ab = alg_bytes(eng.n, D, eng.pat.nnz)
    peak, peak_kind = load_peaks()
    achieved = ab[dom] / (split[dom] * 1e-3) / 1e9
    if rank == 0:
        line = {
            "metric": METRIC, "value": 1000.0 / ms, "unit": "VI iters/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "precision": f"{eng.precision} (FP64 factorisations)",
            "config": {
                "workload": f"{args.workload}: {desc}",
                "schedule": "fused batch VI (block_size=N) on the kNN candidate pattern, kernels sharded over ranks",
                "nnz_pairs": pattern.nnz, "sparsity_threshold": thr,
                "l2": "flushed (256 MB write) before every timed step",
                "parallelism": f"{world} rank(s), kernel rows split by pair count; per-point normaliser all-reduced",
                "init_s": round(t_init, 3), "rank0_kernels": eng.n,
            },
            "roofline": {
                "kernel": dom, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": None, "peak_source": f"{peak_kind} hbm_gbs",
                "alg_bytes_per_launch": ab[dom], "kernel_ms_rank0": {k_: round(v, 4) for k_, v in split.items()},
            },
            "log_pred_density": {"value": len(Xte) / (lpd_ms * 1e-3), "unit": "pts/s", "ms": lpd_ms,
                                 "queries": len(Xte), "kernels": N, "mean_log_density": float(lpd.mean())},
            "e2e": {"value": 1000.0 / e2e_ms, "unit": "VI iters/s", "h2d_bytes_per_step": X.numel() * 4,
                    "d2h_bytes_per_step": 8, "elbo": elbo},
            "gpu_launches": (7 if D > 8 else 5) * args.steps,
            "clocks": clocks.summary(),
            "cpu_baseline": None,
        }
        print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="bsds63", choices=sorted(WORKLOADS))
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64-check", action="store_true", help="skip the mixed / FP32 / FP64 held-out comparison")
    ap.add_argument("--precision", default="auto", choices=["auto", "mixed", "fp32"])
    ap.add_argument("--sharded", action="store_true", help="the sharded engine also with one GPU")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        run_reference(args)
        return

    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", device_id=dev, timeout=datetime.timedelta(seconds=600))
    if world > 1 or args.sharded:
        run_sharded(args, world, rank, dev)
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        return

    if args.workload == "embed43":
        run_hier(args, dev, local)
    else:
        run_single(args, dev, local)


def roofline_fields(durations, N, D, nnz, workload, precision):
    """Roofline of the dominant kernel (HBM: algorithmic bytes / event time
    against the measured copy bandwidth) and the tensor-core kernels' rates."""
    dom = max(durations, key=durations.get)
    ab = alg_bytes(N, D, nnz)
    peak, peak_kind = load_peaks()
    achieved = ab[dom] / (durations[dom] * 1e-3) / 1e9
    fl = alg_flops(N, D, nnz)
    tflops = {k_: round(fl.get(k_, 0) / (v * 1e-3) / 1e12, 3) for k_, v in durations.items()}
    return {
        "kernel": dom, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
        "frac": achieved / peak, "traffic": load_traffic(dom, workload), "peak_source": f"{peak_kind} hbm_gbs",
        "alg_bytes_per_launch": ab[dom], "kernel_ms": {k_: round(v, 5) for k_, v in durations.items()},
        "kernel_alg_tflops": tflops,
        "kernel_hbm_frac": {k_: round(ab[k_] / (v * 1e-3) / 1e9 / peak, 4) for k_, v in durations.items() if k_ in ab},
    }


def run_single(args, dev, local):
    import torch

    from lakde_b200 import LocalKNearestKDE

    Xtr, Xte, k, thr, desc = make_data(args.workload)
    X = torch.tensor(Xtr, device=dev)
    Y = torch.tensor(Xte, device=dev)
    model = LocalKNearestKDE(k_or_knn_graph=k, fused=True, cuda_graph=False, precision=args.precision)
    t_init = time.perf_counter()
    model.fit(X, iterations=0, sparsity_threshold=thr)
    torch.cuda.synchronize()
    t_init = time.perf_counter() - t_init
    eng = model.engine
    N, D = X.shape
    nnz = eng.pattern.nnz
    for _ in range(args.warmup):
        eng.step()
    torch.cuda.synchronize()
    from lakde_b200.tuning import tune_engine

    tuning = tune_engine(eng)  # the launch choices the model's first fused step would make
    eng.tuning = tuning  # kept: the model's own steps below do not tune again
    snap = eng.snapshot()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)  # > 126 MB L2
    torch.cuda.synchronize()
    clocks = ClockSampler(local).__enter__()

    def busy():
        for _ in range(5):
            eng.step()
        torch.cuda.synchronize()

    clocks.wait_for_samples(3, 30.0, busy)
    n_before = len(clocks.samples)
    total_ms = timed_steps(eng, args.steps, flush, torch)
    torch.cuda.synchronize()
    clocks.wait_for_samples(n_before + 2, 30.0, busy)
    clocks.__exit__(None, None, None)
    durations = kernel_split(eng, max(3, args.steps // 2), flush, torch)
    ms_per_step = total_ms / args.steps
    value = 1000.0 / ms_per_step
    roofline = roofline_fields(durations, N, D, nnz, args.workload, eng.precision)

    # the other precision from the same saved state, the same iterations,
    # timed the same way (the plain FP32 kernels against mixed precision)
    plain = None
    if eng.precision == "mixed" or D > 8:
        n_cmp = max(3, args.steps // 2)
        lpd = {}
        ms = {}
        first = eng.precision
        for prec in (first, "fp32" if first == "mixed" else "mixed"):
            eng.precision = prec
            # one untimed step per precision (its buffers and first launches),
            # then the timed steps from the saved state
            eng.restore(snap)
            eng.step()
            eng.restore(snap)
            ms[prec] = timed_steps(eng, n_cmp, flush, torch) / n_cmp
            lpd[prec] = model.log_pred_density(X, Y).double()
        eng.precision = "fp32"
        plain_split = kernel_split(eng, 3, flush, torch)
        eng.precision = first
        eng.restore(snap)
        plain = {
            "value": 1000.0 / ms["fp32"], "unit": "VI iters/s", "ms_per_step": ms["fp32"],
            "kernel_ms": {k_: round(v, 4) for k_, v in plain_split.items()},
            "mixed_value": 1000.0 / ms["mixed"],
            "mixed_speedup": ms["fp32"] / ms["mixed"],
            "held_out_mean_log_density": {
                "iterations_from_same_state": n_cmp,
                "mixed": float(lpd["mixed"].mean()), "plain_fp32": float(lpd["fp32"].mean()),
                "abs_diff_nats": float((lpd["mixed"].mean() - lpd["fp32"].mean()).abs()),
                "max_abs_diff_per_query": float((lpd["mixed"] - lpd["fp32"]).abs().max()),
            },
        }
        del lpd

    # log_pred_density throughput (queries resident in HBM)
    for _ in range(2):
        model.log_pred_density(X, Y)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    lpd_reps = 3
    e0.record()
    for _ in range(lpd_reps):
        lpd = model.log_pred_density(X, Y)
    e1.record()
    torch.cuda.synchronize()
    lpd_ms = e0.elapsed_time(e1) / lpd_reps
    lpd_pts = len(Xte) / (lpd_ms * 1e-3)

    # end to end through the public API with host buffers: pinned X copied into
    # the device buffer the model reads, one partial_step_, ELBO read back
    Xh = torch.tensor(Xtr).pin_memory()
    assert eng.X.data_ptr() == X.data_ptr()
    torch.cuda.synchronize()
    e2e_ms = 0.0
    for _ in range(args.steps):
        flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        X.copy_(Xh, non_blocking=True)
        model.partial_step_(X, 0, sparsity_threshold=thr)
        elbo = float(model.compute_elbo(X))
        b.record()
        torch.cuda.synchronize()
        e2e_ms += a.elapsed_time(b)
    e2e_ms /= args.steps
    model.check_errors_()

    # the host pattern and prior of a sample of rows for the CPU baseline
    cpu_src = None
    if not args.no_cpu_baseline:
        p = eng.pattern
        cpu_src = (p.rowptr.cpu().numpy(), p.col.cpu().numpy(), p.order.cpu().numpy())
        n_keep = min(N, 40_000 if D > 32 else 400_000)
        keep_rows = torch.as_tensor(cpu_src[2][:n_keep].astype(np.int64), device=dev)
        cpu_prior = (eng.sigma_0[keep_rows].cpu().numpy(), eng.sigma_0_tril[keep_rows].cpu().numpy())
        cpu_pos = {int(r_): i for i, r_ in enumerate(cpu_src[2][:n_keep])}
    graph = model.knn_graph
    precision = eng.precision
    gpu_launches = (2 if (D <= 8 and precision == "fp32") else 4) * args.steps
    del model, eng, snap, X, Y, lpd
    torch.cuda.empty_cache()

    check = None
    if not args.no_fp64_check:
        check = fp64_check(Xtr, Xte, graph, thr, 10, dev)

    cpu = None
    if cpu_src is not None:
        def sigma0_fn(rows):
            idx = np.array([cpu_pos[int(r_)] for r_ in rows])
            return cpu_prior[0][idx], cpu_prior[1][idx]

        cpu = cpu_baseline(Xtr, pattern_rows_source(*cpu_src), sigma0_fn, N, nnz, k, thr, float(D))

    line = {
        "metric": METRIC,
        "value": value,
        "unit": "VI iters/s",
        "n_gpus": 1,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_per_step,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "precision": (f"{precision}: tensor-core tf32 hi / lo contractions, FP64 factorisations"
                      if precision == "mixed" else "fp32: plain FP32 GPU kernels, FP64 factorisations"),
        "config": {
            "workload": f"{args.workload}: {desc}",
            "schedule": "fused batch VI (block_size=N) on the kNN candidate pattern",
            "nnz_pairs": nnz,
            "sparsity_threshold": thr,
            "l2": "flushed (256 MB write) before every timed step",
            "parallelism": "single GPU",
            "init_s": round(t_init, 3),
            "launch_choices": tuning,
        },
        "roofline": roofline,
        "plain_fp32": plain,
        "fp64_check": check,
        "log_pred_density": {"value": lpd_pts, "unit": "pts/s", "ms": lpd_ms, "queries": len(Xte),
                             "kernels": N, "precision": precision},
        "e2e": {"value": 1000.0 / e2e_ms, "unit": "VI iters/s", "h2d_bytes_per_step": int(Xtr.size * 4),
                "d2h_bytes_per_step": 8, "elbo": elbo},
        "gpu_launches": gpu_launches,
        "clocks": clocks.summary(),
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)


def run_hier(args, dev, local):
    """LocalHierarchicalKDE, fused, on the near-singular embedded mixture with
    lognormal neighbourhoods (each point explained by its first c_m nearest
    kernels, c_m lognormal, median 64, sigma 1, cap 4,096): the step is one VI
    iteration including the shared-precision update (weighted Gram sum in
    FP64 and its factorisation).  The FP64 check fits mixed, plain FP32 and
    FP64 for 10 iterations (CUDA-graph replay) from the same initialisation."""
    import torch

    from lakde_b200 import LocalHierarchicalKDE
    from lakde_b200 import synthetic as syn
    from lakde_b200.sparse_util import PairPattern
    from lakde_b200.tuning import tune_engine
    from lakde_b200.utils import compute_knn_graph

    Xtr, Xte, k0, thr, desc = make_data(args.workload)
    N, D = Xtr.shape
    X64 = torch.tensor(Xtr.astype(np.float64), device=dev)
    Y64 = torch.tensor(Xte.astype(np.float64), device=dev)
    counts = np.clip(syn.lognormal_neighbourhood_sizes(N, seed=0), k0, N - 1)
    graph = compute_knn_graph(X64, int(counts.max())).long()
    pattern = PairPattern.from_knn_counts(graph, torch.tensor(counts, device=dev))
    seed_graph = graph[:, :k0].to(torch.int32).contiguous()
    del graph

    def make(prec, replay):
        return LocalHierarchicalKDE(k_or_knn_graph=seed_graph, fused=True, candidates=pattern, cuda_graph=replay,
                                    precision=prec)

    X, Y = X64.float(), Y64.float()
    model = make(args.precision, False)
    t_init = time.perf_counter()
    model.fit(X, iterations=0, sparsity_threshold=thr)
    torch.cuda.synchronize()
    t_init = time.perf_counter() - t_init
    eng = model.engine
    nnz = eng.pattern.nnz
    for _ in range(args.warmup):
        eng.step()
    torch.cuda.synchronize()
    tuning = tune_engine(eng)
    eng.tuning = tuning
    snap = eng.snapshot()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    torch.cuda.synchronize()
    clocks = ClockSampler(local).__enter__()

    def busy():
        for _ in range(5):
            eng.step()
        torch.cuda.synchronize()

    clocks.wait_for_samples(3, 30.0, busy)
    n_before = len(clocks.samples)
    eng.restore(snap)
    total_ms = timed_steps(eng, args.steps, flush, torch)
    torch.cuda.synchronize()
    clocks.wait_for_samples(n_before + 2, 30.0, busy)
    clocks.__exit__(None, None, None)
    durations = kernel_split(eng, max(3, args.steps // 2), flush, torch)
    ms_per_step = total_ms / args.steps
    roofline = roofline_fields(durations, N, D, nnz, args.workload, eng.precision)

    # the other precision from the same saved state (one untimed step each)
    n_cmp = max(3, args.steps // 2)
    first = eng.precision
    ms = {}
    for prec in (first, "fp32" if first == "mixed" else "mixed"):
        eng.precision = prec
        eng.restore(snap)
        eng.step()
        eng.restore(snap)
        ms[prec] = timed_steps(eng, n_cmp, flush, torch) / n_cmp
    eng.precision = "fp32"
    plain_split = kernel_split(eng, 3, flush, torch)
    eng.precision = first
    eng.restore(snap)
    plain = {"value": 1000.0 / ms["fp32"], "unit": "VI iters/s", "ms_per_step": ms["fp32"],
             "kernel_ms": {k_: round(v, 4) for k_, v in plain_split.items()},
             "mixed_value": 1000.0 / ms["mixed"], "mixed_speedup": ms["fp32"] / ms["mixed"]}

    # log_pred_density throughput (queries resident in HBM)
    for _ in range(2):
        model.log_pred_density(X, Y)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(3):
        model.log_pred_density(X, Y)
    e1.record()
    torch.cuda.synchronize()
    lpd_ms = e0.elapsed_time(e1) / 3

    # end to end through the public API with host buffers
    Xh = torch.tensor(Xtr).pin_memory()
    assert eng.X.data_ptr() == X.data_ptr()
    e2e_ms = 0.0
    for _ in range(args.steps):
        flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        X.copy_(Xh, non_blocking=True)
        model.partial_step_(X, 0, sparsity_threshold=thr)
        elbo = float(model.compute_elbo(X))
        b.record()
        torch.cuda.synchronize()
        e2e_ms += a.elapsed_time(b)
    e2e_ms /= args.steps
    model.check_errors_()
    precision = eng.precision
    del model, eng, snap
    torch.cuda.empty_cache()

    check = None
    if not args.no_fp64_check:
        res = {}
        for name, dt, prec in (("fp64", torch.float64, "fp32"), ("plain_fp32", torch.float32, "fp32"),
                               ("mixed", torch.float32, "mixed")):
            m = make(prec, True)
            m.fit(X64.to(dt), iterations=10, sparsity_threshold=thr)
            m.check_errors_()
            res[name] = {"mean_log_density": float(m.log_pred_density(X64.to(dt), Y64.to(dt)).double().mean()),
                         "elbo": float(m.compute_elbo(X64.to(dt)))}
            del m
            torch.cuda.empty_cache()
        f = res["fp64"]["mean_log_density"]
        check = {"iterations": 10, "queries": len(Xte), **res,
                 "mixed_vs_fp64_nats": abs(res["mixed"]["mean_log_density"] - f),
                 "plain_fp32_vs_fp64_nats": abs(res["plain_fp32"]["mean_log_density"] - f)}

    line = {
        "metric": METRIC,
        "value": 1000.0 / ms_per_step,
        "unit": "VI iters/s",
        "n_gpus": 1,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_per_step,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "precision": (f"{precision}: tensor-core tf32 hi / lo contractions, FP64 factorisations"
                      if precision == "mixed" else "fp32: plain FP32 GPU kernels, FP64 factorisations"),
        "config": {
            "workload": f"{args.workload}: {desc}",
            "schedule": "fused batch VI (block_size=N) on the lognormal-neighbourhood candidate pattern",
            "nnz_pairs": nnz,
            "sparsity_threshold": thr,
            "l2": "flushed (256 MB write) before every timed step",
            "parallelism": "single GPU",
            "init_s": round(t_init, 3),
            "launch_choices": tuning,
        },
        "roofline": roofline,
        "plain_fp32": plain,
        "fp64_check": check,
        "log_pred_density": {"value": len(Xte) / (lpd_ms * 1e-3), "unit": "pts/s", "ms": lpd_ms,
                             "queries": len(Xte), "kernels": N, "precision": precision},
        "e2e": {"value": 1000.0 / e2e_ms, "unit": "VI iters/s", "h2d_bytes_per_step": int(Xtr.size * 4),
                "d2h_bytes_per_step": 8, "elbo": elbo},
        # M-step, factorisation, E-step, normaliser, weighted Gram sum, shared factorisation
        "gpu_launches": 6 * args.steps,
        "clocks": clocks.summary(),
        "cpu_baseline": None,
    }
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
