"""Benchmark: SDPs/sec to a 1e-7 relative gap on the batched MaxCut workload.

Workload (one "step"): solve a batch of 4096 MaxCut SDP relaxations (seeds
0..4095 per rank, n ~ U{20..120}, G(n, p ~ U(0.05, 0.3)), edge weights
U(0, 1), one n x n block, m = n) to SDPA's pdOPT stopping test with
epsilonStar = 1e-7, inputs resident in HBM.  The headline step is the warm
start and the solve: the low-rank factor of every instance (mixing-method
kernel) and the persistent solver from the SDPAB_INIT_FACTOR start (--start
factor, default), or the learned network's proposal and the solver (--start
learned), or the solver alone from the standard start (--start none).  The
plain FP64 solve from the standard start is timed in the same run.
Synthetic seeded data (no public suite is named).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--precision fp64|mixed] [--start factor|learned|none]
                    [--count C] [--workload maxcut|blocks]

--workload blocks measures the batched multi-block family instead (one GPU,
FP64, standard start): per seed 2..4 SDP blocks of order U{6..40} and an LP
block of U{0..12} entries, m ~ U{10..80}, laid along the diagonal of one
matrix per instance.

Multi-GPU (torchrun): each rank solves its own 4096 instances (independent
units, no collective in the data path): weak scaling; the timed region is the
max over ranks of the device time.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "SDPs/sec to 1e-7 rel gap on 1 B200: mixed+warm-start vs plain FP64"
WORKLOAD = "batched MaxCut: 4096 SDPs, n~U{20..120}, G(n,p~U(0.05,0.3)), w~U(0,1), m=n, eps*=1e-7"
BLOCK_METRIC = "SDPs/sec to 1e-7 rel gap on 1 B200: batched multi-block SDPs, FP64"
BLOCK_WORKLOAD = ("batched multi-block SDPs: 4096 instances, 2..4 SDP blocks of order U{6..40} + LP block "
                  "U{0..12}, m~U{10..80}, eps*=1e-7")


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d["hbm_gbs"], d["bf16_tflops"], "measured"
    return 6650.0, 1590.0, "fallback"


# DRAM bytes (read + write) of the headline solver launch (factor start,
# mixed precision, 4096 instances, 3.18 iterations), from one ncu capture of
# that launch (profiles/batch_ipm_headline_maxcut4096.md): 14.28 GB read +
# 17.00 GB written.  Other batch sizes are scaled by instances.
TRAFFIC_BYTES_HEADLINE = 31.28e9
TRAFFIC_COUNT = 4096
TRAFFIC_NOTE = ("ncu dram__bytes_read.sum + dram__bytes_write.sum of the 4096-instance headline solver launch "
                "(factor start, mixed), profiles/batch_ipm_headline_maxcut4096.md")


def iter_flops(n: int, m: int) -> float:
    """Algorithmic flops of one IPM iteration in the reference's operation
    sequence for one dense block with single-entry constraints (F3 Schur):
    m^3/3 (Schur Cholesky) + 4m^2 (2 solves x 2 trsv) + 8n^3 (dX, pred+corr)
    + 4n^3 (corrector dX dZ Z^-1) + 5n^3/3 (X, Z factor/inverse, Z^-1)
    + Lanczos 2 * k * 4n^2 with k = min(n, ceil(sqrt n) + 10)
      (n <= 20: 2 * (4n^3 + 4n^3/3) for the dense eigenvalue path)
    + F3 assembly 8 m(m+1)/2.  The X D Z^-1 product of dual-infeasible
    iterations (4n^3) is not counted, so this is a lower bound."""
    if n > 20:
        k = min(n, math.ceil(math.sqrt(n)) + 10)
        lan = 2 * k * 4 * n * n
    else:
        lan = 2 * (4 * n ** 3 + 4 * n ** 3 / 3)
    return m ** 3 / 3 + 4 * m * m + 8 * n ** 3 + 4 * n ** 3 + 5 * n ** 3 / 3 + lan + 8 * m * (m + 1) / 2


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = tempfile.mktemp(suffix=".csv")

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            self.proc.wait()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            for line in open(self.path):
                t = [x.strip() for x in line.split(",")]
                if len(t) < 9:
                    continue
                try:
                    sm.append(float(t[1]))
                    mx = max(mx, float(t[2]))
                except ValueError:
                    continue
                for nm, v in zip(names, t[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(nm)
        except OSError:
            pass
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def make_batch(count: int, seed0: int, workload: str = "maxcut"):
    from sdpa_b200 import batch, instances
    gen = instances.batch_block_sdp if workload == "blocks" else instances.batch_maxcut
    insts = [gen(s) for s in range(seed0, seed0 + count)]
    return insts, batch.pack(insts)


def cpu_reference(insts, procs: int, tight: bool = False):
    """The reference solver (oracle/_ref/ref_batch, compiled from the reference
    sources) on every instance of the batch, one single-threaded process per
    core.  Returns (SDPs/s over the slowest worker's summed solve time,
    detail, RefRun with per-instance objectives and x, RefRun at epsilonStar
    1e-11 or None)."""
    from oracle import ref_runner as R
    if not R.available():
        return None, "oracle/_ref/ref_batch not built", None, None
    import shutil
    tmp = tempfile.mkdtemp()
    try:
        R.write_instances(insts, tmp)
        run = R.run(procs=procs, tmp=tmp, count=len(insts))
        trun = R.run(procs=procs, tmp=tmp, count=len(insts), param=R.PARAM_TIGHT) if tight else None
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    det = {"solve_wall_s": run.wall_s, "process_wall_s": run.process_wall_s,
           "pdOPT": int(np.sum(run.phase == 7)), "mean_iterations": float(run.iterations.mean())}
    return len(insts) / run.wall_s, det, run, trun


def run_reference(args):
    """The reference arm: the reference's own CPU solver on the whole batch
    (all `count` instances every step), one single-threaded process per host
    core.  Under torchrun only rank 0 runs."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from oracle import ref_runner as R
    if not R.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/ref_batch is not built"}), flush=True)
        return 0
    insts, _ = make_batch(args.count, 0, args.workload)
    cores = os.cpu_count() or 1
    import shutil
    tmp = tempfile.mkdtemp()
    try:
        R.write_instances(insts, tmp)
        for _ in range(args.warmup):
            R.run(procs=cores, tmp=tmp, count=len(insts))
        runs = [R.run(procs=cores, tmp=tmp, count=len(insts)) for _ in range(args.steps)]
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    walls = [r.wall_s for r in runs]
    value = args.count / float(np.mean(walls))
    last = runs[-1]
    blocks = args.workload == "blocks"
    det = {"solve_wall_s_mean": float(np.mean(walls)), "process_wall_s_mean": float(np.mean([r.process_wall_s for r in runs])),
           "pdOPT": int(np.sum(last.phase == 7)), "mean_iterations": float(last.iterations.mean())}
    line = {"impl": "reference", "metric": BLOCK_METRIC if blocks else METRIC, "value": value, "unit": "SDPs/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * float(np.mean(walls)), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator)",
            "config": {"workload": BLOCK_WORKLOAD if blocks else WORKLOAD, "count": args.count},
            "cpu_baseline": {"value": value, "unit": "SDPs/s", "cores": cores, "kind": "reference",
                             "sample": f"all {args.count} instances of the batch every step, one "
                                       f"single-threaded reference process per core; {det}"},
            "e2e": {"value": value, "unit": "SDPs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def fp64_peak():
    """Measured FP64 GEMM throughput of this GPU (TFLOP/s): torch.matmul on
    float64 8192^3 (cuBLAS DGEMM on the FP64 tensor cores), best of 5 after a
    warm-up, CUDA events.  The batched solver's products run on the same FP64
    MMA and its other steps on the FP64 SIMT pipe."""
    import torch
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    c = torch.empty_like(a)
    torch.matmul(a, b, out=c)
    torch.cuda.synchronize()
    best = 1e30
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b, out=c)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b, c
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / (best / 1e3) / 1e12


def fixed_shape(args) -> dict:
    """The launch shape given on the command line (0 = the library default)."""
    return {"ctas_per_sm": args.ctas_per_sm, "block_threads": args.block_threads}


def _events_time(fn, stream, steps, flush):
    """Device time (ms) of fn() per step, CUDA events on `stream`, L2 flushed
    (256 MB written) before every step."""
    import torch
    times = []
    for _ in range(steps):
        flush.add_(1.0)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    return times


def _capture(fn, stream):
    """CUDA graph of fn() on `stream` (None if capture is not possible)."""
    import torch
    try:
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=stream, capture_error_mode="relaxed"):
            fn()
        return g
    except Exception as e:  # capture unsupported: run eagerly
        print(f"graph capture failed ({e}); timing eager launches", file=sys.stderr)
        return None


def run_blocks(args):
    """The batched multi-block family on one GPU: FP64 from the standard
    start (the reference's own path), one persistent launch per step."""
    import torch
    from sdpa_b200 import _native as N
    from sdpa_b200 import autotune, batch
    if int(os.environ.get("WORLD_SIZE", "1")) > 1:
        raise SystemExit("--workload blocks runs on one GPU")
    torch.cuda.set_device(0)
    insts, P = make_batch(args.count, 0, "blocks")
    db = batch.DeviceBatch(P)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    stream = torch.cuda.Stream()
    cand = [fixed_shape(args)] if (args.ctas_per_sm > 0 or args.block_threads > 0) else None
    tune = autotune.tune(db, N.PREC_FP64, stream=stream, candidates=cand)
    c = tune["best"]
    run = lambda: db.solve(precision=N.PREC_FP64, stream=stream, **c)
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            run()
        torch.cuda.synchronize()
        with ClockSampler(0) as clk:
            times = _events_time(run, stream, args.steps, flush)
    torch.cuda.synchronize()
    res = db.result()
    step_ms = float(np.mean(times))
    value = P.count / (step_ms / 1e3)
    # e2e: host (pinned) inputs -> device, solve, results -> host
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
    pairs = [(db.d[k], pin(getattr(P, k))) for k in db.d] + [(db.order, pin(db.order.cpu().numpy()))]
    h2d = sum(h.numel() * h.element_size() for _, h in pairs)
    out_sc = torch.empty_like(db.sc, device="cpu").pin_memory()
    out_ic = torch.empty_like(db.ic, device="cpu").pin_memory()
    out_x = torch.empty_like(db.xvec, device="cpu").pin_memory()
    d2h = out_sc.numel() * 8 + out_ic.numel() * 4 + out_x.numel() * 8
    e2e_t = []
    for _ in range(max(1, min(args.steps, 3))):
        flush.add_(1.0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        with torch.cuda.stream(stream):
            for dev, host in pairs:
                dev.copy_(host, non_blocking=True)
            run()
            out_sc.copy_(db.sc, non_blocking=True)
            out_ic.copy_(db.ic, non_blocking=True)
            out_x.copy_(db.xvec, non_blocking=True)
        stream.synchronize()
        e2e_t.append(time.perf_counter() - t0)
    line = {"metric": BLOCK_METRIC, "value": value, "unit": "SDPs/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator, no public suite)",
            "config": {"workload": BLOCK_WORKLOAD, "count_per_gpu": args.count, "precision": "fp64",
                       "warm_start": False, "launch_shape": c, "autotune_ms": tune["ms"],
                       "l2": "256 MB buffer written between timed steps", "parallelism": "replicas x1"},
            "e2e": {"value": P.count / float(np.mean(e2e_t)), "unit": "SDPs/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h)},
            "gpu_launches": args.steps, "clocks": clk.summary(),
            "parity": {"pdOPT": int(np.sum(res.phase == 7)), "count": int(P.count),
                       "mean_iterations": float(res.iterations.mean()), "status_nonzero": int(np.sum(res.status != 0))}}
    if not args.no_cpu_baseline:
        cores = os.cpu_count() or 1
        v, det, ref, tref = cpu_reference(insts, cores, tight=True)
        line["cpu_baseline"] = {"value": v, "unit": "SDPs/s", "cores": cores, "kind": "reference",
                                "sample": f"all {P.count} instances of this batch, one single-threaded "
                                          f"reference process per core; {det}"}
        if ref is not None:
            from oracle import ref_runner as R
            line["reference_parity"] = R.parity_counts(res.primal_obj, res.dual_obj,
                                                       [res.x_of(P, q) for q in range(P.count)], ref, tref,
                                                       phase=res.phase)
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed"])
    ap.add_argument("--start", default="factor", choices=["factor", "learned", "none"],
                    help="headline start: low-rank factor (mixing method + SDPAB_INIT_FACTOR), the learned "
                         "network's proposal (SDPAB_INIT_DUAL), or the standard start")
    ap.add_argument("--warm", type=int, default=None, help="0: same as --start none (kept for old commands)")
    ap.add_argument("--count", type=int, default=4096)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-graph", action="store_true")
    ap.add_argument("--ctas-per-sm", type=int, default=0, help="fixed launch shape (0 = autotune)")
    ap.add_argument("--block-threads", type=int, default=0, help="fixed threads per instance, 256 or 128 (0 = autotune)")
    ap.add_argument("--workload", default="maxcut", choices=["maxcut", "blocks"])
    ap.add_argument("--profile", action="store_true",
                    help="only launch the headline pipeline warmup + steps times, untimed (for ncu captures)")
    args = ap.parse_args()
    if args.warm == 0:
        args.start = "none"
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "blocks":
        return run_blocks(args)

    import torch
    import torch.distributed as dist
    from sdpa_b200 import _native as N
    from sdpa_b200 import autotune, batch, lowrank
    from sdpa_b200 import warmstart as W

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    prec = N.PREC_FP64 if args.precision == "fp64" else N.PREC_MIXED

    seed0 = rank * args.count
    graphs = [W.batch_graph(s, 20, 120) for s in range(seed0, seed0 + args.count)]
    insts = [g.instance() for g in graphs]
    P = batch.pack(insts)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    stream = torch.cuda.Stream()

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()

    def make_pipe(start, db):
        if start == "factor":
            return lowrank.FactorPipeline(db)
        if start == "learned":
            return W.WarmPipeline(W.default_model(), graphs, db)
        return None

    if args.profile:
        # the headline pipeline alone, launched warmup + steps times (one
        # solver launch each), for a profiler: nothing is timed or printed
        # but the instances' outcome
        dbp = batch.DeviceBatch(P)
        pp = make_pipe(args.start, dbp)
        for _ in range(args.warmup + args.steps):
            if pp is not None:
                pp.run(precision=prec, stream=stream, **fixed_shape(args))
            else:
                dbp.solve(precision=prec, stream=stream, **fixed_shape(args))
        barrier()
        r = dbp.result()
        if rank == 0:
            print(json.dumps({"profile": True, "count": args.count, "launches": args.warmup + args.steps,
                              "pdOPT": int(np.sum(r.phase == 7)), "mean_iterations": float(r.iterations.mean())}))
        if world > 1:
            dist.destroy_process_group()
        return 0

    # ---- plain FP64 path (standard start): the denominator of the headline ratio
    db0 = batch.DeviceBatch(P)
    cand = [fixed_shape(args)] if (args.ctas_per_sm > 0 or args.block_threads > 0) else None
    tune0 = autotune.tune(db0, N.PREC_FP64, stream=stream, candidates=cand)
    c0 = tune0["best"]
    run0 = lambda: db0.solve(precision=N.PREC_FP64, stream=stream, **c0)
    # ---- headline path: precision + warm start
    dbh = batch.DeviceBatch(P)
    pipe = make_pipe(args.start, dbh)
    tuneh = autotune.tune(dbh, prec, stream=stream, candidates=cand,
                          run=(lambda c: pipe.run(precision=prec, stream=stream, **c)) if pipe else None)
    ch = tuneh["best"]
    if pipe is not None:
        runh = lambda: pipe.run(precision=prec, stream=stream, **ch)
    else:
        runh = lambda: dbh.solve(precision=prec, stream=stream, **ch)

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            run0()
            runh()
    barrier()
    g0 = gh = None
    if not args.no_graph:
        g0 = _capture(run0, stream)
        gh = _capture(runh, stream)
    step0 = (lambda: g0.replay()) if g0 is not None else run0
    steph = (lambda: gh.replay()) if gh is not None else runh
    with torch.cuda.stream(stream):
        step0()
        steph()
    barrier()

    with torch.cuda.stream(stream):
        t_plain = _events_time(step0, stream, args.steps, flush)
        barrier()
        with ClockSampler(local) as clk:
            times = _events_time(steph, stream, args.steps, flush)
        barrier()
    # the pipeline's two stages timed apart (factor: the mixing kernel;
    # solve: the persistent solver from the start), and the learned network's
    # start in the same precision, same batch, same timing
    stages = None
    if isinstance(pipe, lowrank.FactorPipeline):
        with torch.cuda.stream(stream):
            tf = _events_time(lambda: pipe.factor(stream), stream, args.steps, flush)
            ts = _events_time(lambda: dbh.solve(precision=prec, stream=stream, **ch), stream, args.steps, flush)
        barrier()
        stages = {"factor_ms": float(np.mean(tf)), "solve_ms": float(np.mean(ts)),
                  "mean_sweeps": float(pipe.sweeps.float().mean().item()),
                  "max_sweeps": int(pipe.sweeps.max().item())}
    alt = None
    if args.start != "learned":
        dbl = batch.DeviceBatch(P)
        lp = W.WarmPipeline(W.default_model(), graphs, dbl)
        ach = {k: v for k, v in ch.items() if k != "mixed_products"}
        with torch.cuda.stream(stream):
            for _ in range(2):
                lp.run(precision=prec, stream=stream, **ach)
            ta = _events_time(lambda: lp.run(precision=prec, stream=stream, **ach), stream, args.steps, flush)
        barrier()
        ra = dbl.result()
        alt = {"start": "learned network proposal (SDPAB_INIT_DUAL)", "precision": args.precision,
               "value": args.count / (float(np.mean(ta)) / 1e3), "unit": "SDPs/s (this GPU)",
               "ms_per_step": float(np.mean(ta)), "mean_iterations": float(ra.iterations.mean()),
               "pdOPT": int(np.sum(ra.phase == 7)), "retried_in_fp64": int(np.sum(ra.status == 2))}
        del lp, dbl
    with torch.cuda.stream(stream):
        steph()
    barrier()
    res = dbh.result()
    res0 = db0.result()
    step_ms = float(np.mean(times))
    plain_ms = float(np.mean(t_plain))
    t = torch.tensor([step_ms, plain_ms], device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    step_ms_max, plain_ms_max = float(t[0].item()), float(t[1].item())
    total = args.count * world
    value = total / (step_ms_max / 1e3)
    plain_value = total / (plain_ms_max / 1e3)

    # ---- e2e: host (pinned) inputs -> device, the same pipeline, results -> host
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
    pairs = [(dbh.d[k], pin(getattr(P, k))) for k in dbh.d]
    pairs.append((dbh.order, pin(dbh.order.cpu().numpy())))
    if isinstance(pipe, W.WarmPipeline):
        gb = pipe.dg.gb
        pairs += [(pipe.dg.rowptr, pin(gb.rowptr)), (pipe.dg.col, pin(gb.col)), (pipe.dg.aval, pin(gb.aval)),
                  (pipe.dg.aval_t, pin(gb.aval_t)), (pipe.dg.feat, pin(gb.feat)),
                  (pipe.degree, pin(pipe.degree.cpu().numpy())), (pipe.fallback, pin(pipe.fallback.cpu().numpy()))]
    h2d = sum(h.numel() * h.element_size() for _, h in pairs)
    out_sc = torch.empty_like(dbh.sc, device="cpu").pin_memory()
    out_ic = torch.empty_like(dbh.ic, device="cpu").pin_memory()
    out_x = torch.empty_like(dbh.xvec, device="cpu").pin_memory()
    d2h = out_sc.numel() * 8 + out_ic.numel() * 4 + out_x.numel() * 8
    e2e_t = []
    for _ in range(max(1, min(args.steps, 3))):
        flush.add_(1.0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        with torch.cuda.stream(stream):
            for dev, host in pairs:
                dev.copy_(host, non_blocking=True)
            steph()
            out_sc.copy_(dbh.sc, non_blocking=True)
            out_ic.copy_(dbh.ic, non_blocking=True)
            out_x.copy_(dbh.xvec, non_blocking=True)
        stream.synchronize()
        e2e_t.append(time.perf_counter() - t0)
    barrier()
    t = torch.tensor([float(np.mean(e2e_t))], device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    e2e_val = total / float(t.item())

    # ---- roofline of the solver launch: algorithmic flops of the iterations
    # each instance ran (reference operation sequence) / device time, against
    # the measured FP64 GEMM peak (the kernel's products run on the FP64 MMA,
    # the rest on the FP64 / FP32 SIMT pipes) and, for scale, the bf16 peak
    flops = sum(float(res.iterations[q]) * iter_flops(int(P.n[q]), int(P.m[q])) for q in range(P.count))
    hbm, bf16, src = peaks()
    fp64 = fp64_peak()
    # the solver launch's own time when the step also runs the factor kernel
    solver_ms = stages["solve_ms"] if stages else step_ms
    achieved = flops / (solver_ms / 1e3) / 1e12
    traffic = TRAFFIC_BYTES_HEADLINE * P.count / TRAFFIC_COUNT
    # factor: mixing kernel + solver; learned: 7 network + 1 proposal + 1 solver
    launches_per_step = {"factor": 2, "learned": 9, "none": 1}[args.start]
    relobj = np.abs(res.primal_obj - res0.primal_obj) / np.maximum(1.0, np.abs(res0.primal_obj))
    xdiff = np.array([np.max(np.abs(res.x_of(P, q) - res0.x_of(P, q))) for q in range(P.count)])
    line = {"metric": METRIC, "value": value, "unit": "SDPs/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_ms_max, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if prec == N.PREC_FP64 else "f32+f64",
            "data": "synthetic (seeded generator, no public suite)",
            "config": {"workload": WORKLOAD, "count_per_gpu": args.count, "precision": args.precision,
                       "start": {"factor": "low-rank factor (mixing method) + SDPAB_INIT_FACTOR",
                                 "learned": "learned network proposal (SDPAB_INIT_DUAL)",
                                 "none": "standard start lambda* I"}[args.start],
                       "cuda_graph": gh is not None,
                       "launch_shape": {"headline": ch, "plain_fp64": c0, "autotune_ms_headline": tuneh["ms"],
                                        "autotune_ms_plain_fp64": tune0["ms"]},
                       "l2": "256 MB buffer written between timed steps",
                       "parallelism": f"replicas x{world} (independent instances per GPU)"},
            "plain_fp64": {"value": plain_value, "unit": "SDPs/s", "ms_per_step": plain_ms_max,
                           "mean_iterations": float(res0.iterations.mean()),
                           "pdOPT": int(np.sum(res0.phase == 7))},
            "speedup_vs_plain_fp64": value / plain_value,
            "stages": stages,
            "learned_warm_start": alt,
            "e2e": {"value": e2e_val, "unit": "SDPs/s", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
            "gpu_launches": args.steps * launches_per_step,
            "roofline": {"bound": "tensor", "pipe": "FP64 MMA (mma.sync .f64) + FP64/FP32 SIMT",
                         "achieved": achieved, "peak": fp64, "unit": "TFLOP/s", "frac": achieved / fp64,
                         "peak_source": "FP64 GEMM measured in this run (torch.matmul float64 8192^3, "
                                        "cuBLAS DGEMM, best of 5)",
                         "traffic": traffic, "traffic_note": TRAFFIC_NOTE,
                         "bf16_peak": bf16, "frac_of_bf16": achieved / bf16,
                         "bf16_peak_source": f"{src} (MEASURED_PEAKS.json)",
                         "flops_per_launch": flops, "kernel": "batch_ipm_fp64", "kernel_ms": solver_ms},
            "clocks": clk.summary(),
            "parity": {"pdOPT": int(np.sum(res.phase == 7)), "count": int(P.count),
                       "mean_iterations": float(res.iterations.mean()),
                       "retried_in_fp64": int(np.sum(res.status == 2)),
                       "max_rel_objective_diff_vs_plain_fp64": float(relobj.max()),
                       "max_abs_x_diff_vs_plain_fp64": float(xdiff.max()),
                       "x_diff_above_1e-5_vs_plain_fp64": int(np.sum(xdiff > 1e-5))}}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cores = os.cpu_count() or 1
        v, det, ref, tref = cpu_reference(insts, cores, tight=True)
        line["cpu_baseline"] = {"value": v, "unit": "SDPs/s", "cores": cores, "kind": "reference",
                                "sample": f"all {P.count} instances of this batch, one single-threaded "
                                          f"reference process per core; {det}"}
        if ref is not None:
            # the headline run's every instance against the reference's own
            # results on the same input (objectives 1e-6, x 1e-5, and the
            # reference-accuracy bar against its epsilonStar 1e-11 solution)
            from oracle import ref_runner as R
            xs = [res.x_of(P, q) for q in range(P.count)]
            line["reference_parity"] = R.parity_counts(res.primal_obj, res.dual_obj, xs, ref, tref, phase=res.phase)
            xs0 = [res0.x_of(P, q) for q in range(P.count)]
            line["plain_fp64"]["reference_parity"] = R.parity_counts(res0.primal_obj, res0.dual_obj, xs0, ref,
                                                                      phase=res0.phase)
    del g0, gh
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
