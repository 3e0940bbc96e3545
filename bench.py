"""Benchmark of the lakde VI hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload gas8|bsds63|...]
                    [--impl reference]

A step is one VI iteration of LocalKNearestKDE over all N kernels (fused
batch schedule on the kNN candidate pattern), on seeded synthetic data with
the shape of the named workload.  Inputs are resident in HBM; L2 is flushed
between timed steps.  Rank 0 prints one JSON line with the whole-job
throughput, the roofline of the dominant kernel, the end-to-end number
through the public API with host buffers, the CPU baseline (the oracle port
timed on a bounded sample) and the SM clocks sampled during the timed region.
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
    "bsds63s": (dict(n_train=50_000, n_test=1_024), 100, 5e-4,
                "LocalKNearestKDE d=63 N_train=50000 N_test=1024 K=100 (the bsds63 mixture, small case for "
                "profiling)"),
    "spec21": (dict(n_train=300_000, n_test=4_096), 64, 5e-4,
               "LocalKNearestKDE d=21 N_train=300000 N_test=4096 K=64 (12-component mixture)"),
    "circle2d": (dict(n_train=2_000, n_test=1_000), 20, 0.0,
                 "LocalKNearestKDE d=2 N_train=2000 N_test=1000 K=20 (8-Gaussian circle)"),
}


def make_data(name):
    from lakde_b200 import synthetic as syn

    kw, k, thr, desc = WORKLOADS[name]
    gen = {"gas8": syn.heavy_tail_mixture, "bsds63": syn.decaying_spectrum_mixture,
           "bsds63s": syn.decaying_spectrum_mixture,
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
    from lakde_b200 import kernels as K

    stream = torch.cuda.current_stream()
    p = eng.pattern
    if eng.D <= 8:
        launches = {
            "vi_rows": lambda: K.vi_rows(p.rowptr, p.col, eng.r, eng.X, eng.nu_0, eng.a, eng.b, eng.b_0_f,
                                         eng.W_inv_jitter, eng.eps, eng.nu, eng.logdet_W, eng.info, eng.logrho,
                                         P=eng.sigma_0, T=eng.sigma_0_tril, order=p.order,
                                         mm=eng.sigma_0_lambda_mm_trace),
        }
    else:
        tcs = "_tc" if eng.precision == "mixed" else ""
        launches = {"mstep" + tcs: eng.mstep, "posterior_factor": eng.factor,
                    "estep" + (tcs or "_logrho"): eng.estep_numerators}
    launches["estep_normalise"] = lambda: K.estep_normalise(p.cptr, p.pos, eng.logrho, eng.r, eng.c, eng.rsum, 1,
                                                            eng.threshold)
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


def cpu_baseline(Xtr, graph, k, thr, budget_s=20.0):
    """The reference algorithm (oracle port, numpy) timed on a bounded sample of
    one VI iteration of its block schedule (blocks of 512 kernels, dense E-step
    against every point): the posterior of one kernel block, then as many of
    its point blocks of the dense E-step as fit the time budget; extrapolated
    to all point blocks and all kernel blocks."""
    from oracle import lakde_oracle as O

    N, D = Xtr.shape
    B = 512
    m = O.KNNKDEOracle(k=graph.astype(np.int64), block_size=B)
    m.init_parameters_(Xtr, thr)
    m.rnm_log_consts[:] = 0.0
    t0 = time.perf_counter()
    S, nu = m._posterior_contribs(Xtr, 0)
    sigma_0, _ = m.prior_cov(Xtr, 0)
    W = m._posterior(0, N, sigma_0, S)
    t_post = time.perf_counter() - t0
    logdet = O.chol_logdet(W)
    n_pb = (N - 1) // B + 1
    done = 0
    t1 = time.perf_counter()
    while done < n_pb and (done < 1 or time.perf_counter() - t1 < budget_s):
        js = done * B
        lr = O.calc_log_rho_block(Xtr[js:js + B], Xtr[:B], nu, W, logdet)
        c = O.logsumexp0(lr)
        r = np.exp(lr - c[None, :])
        if thr:
            r = np.where(r > thr, r, 0)
        np.nonzero(r)
        done += 1
    t_block = (time.perf_counter() - t1) / done
    per_step = t_post + n_pb * t_block
    n_kb = (N - 1) // B + 1
    return {
        "value": 1.0 / (per_step * n_kb),
        "unit": "VI iters/s",
        "cores": os.cpu_count(),
        "kind": "port",
        "sample": (f"posterior of one 512-kernel block ({t_post:.2f} s) + {done} of {n_pb} point blocks of its "
                   f"dense E-step ({t_block:.3f} s each), numpy oracle; extrapolated to {n_pb} point blocks x "
                   f"{n_kb} kernel blocks"),
    }


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    Xtr, Xte, k, thr, desc = make_data(args.workload)
    from oracle import lakde_oracle as O

    # kNN graph for the sample: exact ranks of the first block's neighbourhoods only
    N = len(Xtr)
    graph = np.empty((N, k), dtype=np.int64)
    rng = np.random.default_rng(0)
    # the sampled steps read the graph rows of their own blocks only; other rows
    # get random neighbours (they do not enter the timed work)
    graph[:] = rng.integers(0, N, size=(N, k))
    graph[:1024] = O.knn_graph(Xtr, k)[:1024] if N <= 1024 else _block_knn(Xtr, k, 1024)
    # each timed step is one bounded sample; stop after ~90 s
    vals = []
    t0 = time.perf_counter()
    for _ in range(max(1, args.steps)):
        vals.append(cpu_baseline(Xtr, graph, k, thr, budget_s=5.0))
        if time.perf_counter() - t0 > 90.0:
            break
    v = statistics.median([x["value"] for x in vals])
    cb = dict(vals[-1])
    cb["value"] = v
    args.steps = len(vals)
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "VI iters/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"{args.workload}: {desc}", "schedule": "block_size=512, dense E-step"},
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
                                      eng.precision, eng.err), reps),
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
            "gpu_launches": 7 * args.steps,
            "clocks": clocks.summary(),
            "cpu_baseline": None,
        }
        print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="gas8", choices=sorted(WORKLOADS))
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
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
    snap = eng.snapshot()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)  # > 126 MB L2

    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local).__enter__()

    def busy():
        for _ in range(20):
            eng.step()
        torch.cuda.synchronize()

    clocks.wait_for_samples(3, 20.0, busy)
    n_before = len(clocks.samples)
    total_ms = timed_steps(eng, args.steps, flush, torch)
    torch.cuda.synchronize()
    clocks.wait_for_samples(n_before + 2, 20.0, busy)
    clocks.__exit__(None, None, None)
    durations = kernel_split(eng, max(3, args.steps // 2), flush, torch)
    ms_per_step = total_ms / args.steps
    if world > 1:
        t = torch.tensor([ms_per_step], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_per_step = float(t)
    value = world * 1000.0 / ms_per_step

    # the roofline of the dominant kernel (HBM: compulsory bytes; the quad
    # forms and the scatter at large D are gathers of whole point rows, so
    # they are bound by memory, not by the tensor pipe)
    dom = max(durations, key=durations.get)
    ab = alg_bytes(N, D, nnz)
    peak, peak_kind = load_peaks()
    achieved = ab[dom] / (durations[dom] * 1e-3) / 1e9
    traffic = load_traffic(dom, args.workload)
    tflops = {k_: alg_flops(N, D, nnz).get(k_, 0) / (v * 1e-3) / 1e12 for k_, v in durations.items()}

    # plain FP32 against mixed precision: the same number of iterations from the
    # same saved state, timed the same way (large D only)
    plain = None
    if D > 8 and eng.precision == "mixed":
        n_cmp = max(3, args.steps // 2)
        lpd = {}
        ms = {}
        for prec in ("mixed", "fp32"):
            eng.restore(snap)
            eng.precision = prec
            ms[prec] = timed_steps(eng, n_cmp, flush, torch) / n_cmp
            lpd[prec] = model.log_pred_density(X, Y).double()
        plain_split = kernel_split(eng, 3, flush, torch)
        eng.precision = "mixed"
        plain = {
            "value": 1000.0 / ms["fp32"], "unit": "VI iters/s", "ms_per_step": ms["fp32"],
            "kernel_ms": {k_: round(v, 4) for k_, v in plain_split.items()},
            "mixed_speedup": ms["fp32"] / ms["mixed"],
            "held_out_mean_log_density": {
                "iterations_from_same_state": n_cmp,
                "mixed": float(lpd["mixed"].mean()), "plain_fp32": float(lpd["fp32"].mean()),
                "abs_diff_nats": float((lpd["mixed"].mean() - lpd["fp32"].mean()).abs()),
                "max_abs_diff_per_query": float((lpd["mixed"] - lpd["fp32"]).abs().max()),
            },
        }

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

    # end to end through the public API with host buffers: pinned X copied
    # into the device buffer the model and its captured iteration read, one
    # partial_step_, ELBO read back to the host
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

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(Xtr, model.knn_graph.cpu().numpy(), k, thr)

    if rank == 0:
        line = {
            "metric": METRIC,
            "value": value,
            "unit": "VI iters/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms_per_step,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic",
            "precision": (f"{eng.precision} (FP64 factorisations)" if D > 8 else
                          "fp32 (plain FP32 GPU kernels; FP64 factorisations)"),
            "config": {
                "workload": f"{args.workload}: {desc}",
                "schedule": "fused batch VI (block_size=N) on the kNN candidate pattern",
                "nnz_pairs": nnz,
                "sparsity_threshold": thr,
                "l2": "flushed (256 MB write) before every timed step",
                "parallelism": "single GPU",
                "init_s": round(t_init, 3),
            },
            "roofline": {
                "kernel": dom,
                "bound": "hbm",
                "achieved": achieved,
                "peak": peak,
                "unit": "GB/s",
                "frac": achieved / peak,
                "traffic": traffic,
                "peak_source": f"{peak_kind} hbm_gbs",
                "alg_bytes_per_launch": ab[dom],
                "kernel_ms": {k_: round(v, 5) for k_, v in durations.items()},
                "kernel_alg_tflops": {k_: round(v, 3) for k_, v in tflops.items()},
            },
            "plain_fp32": plain,
            "log_pred_density": {"value": lpd_pts, "unit": "pts/s", "ms": lpd_ms, "queries": len(Xte),
                                 "kernels": N, "mean_log_density": float(lpd.mean())},
            "e2e": {"value": world * 1000.0 / e2e_ms, "unit": "VI iters/s", "h2d_bytes_per_step": X.numel() * 4,
                    "d2h_bytes_per_step": 8, "elbo": elbo},
            "gpu_launches": (2 if D <= 8 else 4) * args.steps,
            "clocks": clocks.summary(),
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
