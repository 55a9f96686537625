"""Autotuner of the batched solver's launch shape.

The persistent kernel runs one 256-thread block per instance in flight; the
free parameter is how many blocks share an SM (1 or 2 fit the register and
shared-memory budget).  More blocks per SM hide more latency but put more
per-block workspace (15 n^2 doubles each) into L2.  The tuner times every
candidate on the batch itself (device events, after a warm-up) and keeps the
fastest per (nmax class, precision).
"""
from __future__ import annotations

_cache: dict = {}


def size_class(nmax: int) -> int:
    for c in (32, 64, 96, 128, 256, 512):
        if nmax <= c:
            return c
    return 1024


def tune(db, precision: int = 0, candidates=(1, 2), reps: int = 2, run=None, stream=None) -> dict:
    """Time one solve step for each ctas_per_sm candidate; returns {"best": c,
    "ms": {c: ms}} and caches the choice for the batch's size class.  `run(c)`
    issues the step (default: db.solve with that launch shape) on `stream`."""
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    if run is None:
        run = lambda c: db.solve(precision=precision, stream=s, ctas_per_sm=c)
    key = (size_class(db.P.nmax), precision)
    res = {}
    for c in candidates:
        run(c)
        torch.cuda.synchronize()
        best = 1e30
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(s)
            run(c)
            e1.record(s)
            e1.synchronize()
            best = min(best, e0.elapsed_time(e1))
        res[c] = best
    choice = min(res, key=res.get)
    _cache[key] = choice
    return {"best": choice, "ms": res, "class": key[0]}


def choice(nmax: int, precision: int = 0, default: int = 2) -> int:
    return _cache.get((size_class(nmax), precision), default)
