"""Trains the warm-start network on solutions the solver itself produces and
evaluates it on held-out instances.

    python -m sdpa_b200.train_warmstart [--train 20000] [--test 2048] [--epochs 20]
                                        [--out sdpa_b200/data] [--nmin 50 --nmax 200]

Training set: MaxCut SDPs of seeds 100000.. (n ~ U{nmin..nmax}, p ~ U(0.05,
0.3), w ~ U(0,1)), solved by the batched FP64 solver; targets r_i = 4 x_i/d_i.
Held-out set: seeds 300000.., disjoint.  Writes mpnn_maxcut.npy (FP32 master
weights) and mpnn_maxcut_eval.json (iterations, SDPs/s and objective
agreement of warm vs standard start, device-timed).
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from . import _native as N
from . import batch as B
from . import warmstart as W

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_WEIGHTS = os.path.join(HERE, "data", "mpnn_maxcut.npy")


def solve_chunked(graphs, chunk=4096, **kw):
    out = []
    for c0 in range(0, len(graphs), chunk):
        P, r = W.solve_graphs(graphs[c0:c0 + chunk], **kw)
        out.append((P, r))
    return out


def device_timed(graphs, init_x=None, reps=3, precision=N.PREC_FP64):
    """SDPs/s of the device-resident batched solve (CUDA events)."""
    import torch
    P = B.pack([g.instance() for g in graphs])
    db = B.DeviceBatch(P)
    if init_x is not None:
        xv = np.zeros(P.nvec)
        for q, x in enumerate(init_x):
            xv[P.vec_off[q]:P.vec_off[q] + P.m[q]] = x
        db.set_init(np.full(P.count, W.INIT_DUAL, np.int32), xv)
    db.solve(precision=precision)
    torch.cuda.synchronize()
    ts = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        db.solve(precision=precision)
        e1.record()
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1) / 1e3)
    return P, db.result(), P.count / min(ts)


def evaluate(model, graphs, label, precision=N.PREC_FP64):
    import torch
    t0 = time.time()
    x_prop = W.propose_x(model, graphs)
    # network inference time on the device (features already built)
    gb = W.make_graph_batch(graphs)
    dg = W.DeviceGraphs(gb)
    model.forward(dg)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    model.forward(dg)
    e1.record()
    torch.cuda.synchronize()
    infer_s = e0.elapsed_time(e1) / 1e3
    Pc, cold, sps_cold = device_timed(graphs, precision=precision)
    Pw, warm, sps_warm = device_timed(graphs, x_prop, precision=precision)
    relobj = np.abs(warm.primal_obj - cold.primal_obj) / np.maximum(1.0, np.abs(cold.primal_obj))
    xerr = max(float(np.max(np.abs(warm.x_of(Pw, q) - cold.x_of(Pc, q)))) for q in range(Pc.count))
    n = len(graphs)
    return {
        "set": label, "instances": n,
        "cold_iterations_mean": float(cold.iterations.mean()),
        "warm_iterations_mean": float(warm.iterations.mean()),
        "cold_pdOPT": int(np.sum(cold.phase == 7)), "warm_pdOPT": int(np.sum(warm.phase == 7)),
        "warm_fallbacks": int(np.sum(warm.status == 1)),
        "max_rel_objective_diff": float(relobj.max()), "max_abs_x_diff": xerr,
        "cold_sdps_per_s": sps_cold,
        "warm_sdps_per_s_solver_only": sps_warm,
        "warm_sdps_per_s_incl_network": n / (n / sps_warm + infer_s),
        "network_inference_s": infer_s,
        "wall_s": time.time() - t0,
    }


def evaluate_all(model, args):
    """Held-out set and the batched-MaxCut benchmark set, FP64 and mixed."""
    test_g = [W.batch_graph(s, args.nmin, args.nmax) for s in range(300000, 300000 + args.test)]
    mcb = [W.batch_graph(s, 20, 120) for s in range(4096)]
    ev = []
    for prec, name in ((N.PREC_FP64, "fp64"), (N.PREC_MIXED, "mixed")):
        for graphs, label in ((test_g, f"held-out n~U{{{args.nmin}..{args.nmax}}} seeds 300000+"),
                              (mcb, "batched MaxCut n~U{20..120} seeds 0..4095")):
            e = evaluate(model, graphs, label, prec)
            e["precision"] = name
            ev.append(e)
    return ev


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--train", type=int, default=20000)
    ap.add_argument("--test", type=int, default=2048)
    ap.add_argument("--epochs", type=int, default=20)
    ap.add_argument("--batch", type=int, default=256)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--nmin", type=int, default=50)
    ap.add_argument("--nmax", type=int, default=200)
    ap.add_argument("--out", default=os.path.join(HERE, "data"))
    ap.add_argument("--eval-only", action="store_true", help="load mpnn_maxcut.npy and evaluate")
    args = ap.parse_args()
    if args.eval_only:
        model = W.MPNN(seed=0)
        model.load(np.load(DEFAULT_WEIGHTS))
        print(json.dumps({"eval": evaluate_all(model, args)}, indent=1), flush=True)
        return
    os.makedirs(args.out, exist_ok=True)
    t0 = time.time()
    train_g = [W.batch_graph(s, args.nmin, args.nmax) for s in range(100000, 100000 + args.train)]
    sols = solve_chunked(train_g)
    ts, ms = [], []
    for c, (P, r) in enumerate(sols):
        sub = train_g[c * 4096:(c + 1) * 4096]
        t, m = W.targets_from_solution(sub, P, r)
        ts.append(t)
        ms.append(m)
    targets, masks = np.concatenate(ts), np.concatenate(ms)
    ok = int(sum(int(np.sum(r.phase == 7)) for _, r in sols))
    print(f"training data: {args.train} solves ({ok} pdOPT) in {time.time() - t0:.1f}s", flush=True)
    model = W.MPNN(seed=0)
    t1 = time.time()
    hist = W.train(model, train_g, targets, masks, epochs=args.epochs, batch_graphs=args.batch, lr=args.lr,
                   log=lambda s: print(s, flush=True))
    train_s = time.time() - t1
    np.save(os.path.join(args.out, "mpnn_maxcut.npy"), model.state())
    ev = evaluate_all(model, args)
    summary = {"train_instances": args.train, "train_pdOPT": ok, "epochs": args.epochs,
               "loss_first_epoch": hist[0], "loss_last_epoch": hist[-1], "train_seconds": train_s,
               "params": model.P, "eval": ev}
    with open(os.path.join(args.out, "mpnn_maxcut_eval.json"), "w") as f:
        json.dump(summary, f, indent=1)
    print(json.dumps(summary, indent=1), flush=True)


if __name__ == "__main__":
    main()
