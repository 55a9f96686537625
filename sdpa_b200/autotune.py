"""Autotuner of the batched solver's launch shape.

The persistent kernel runs one instance per block of threads; the shape
decides how its dense steps map onto the SM:

* block_threads: 256 threads (8 warps) per instance, two blocks per SM, the
  square products on one exact-size FP64-MMA tile (n <= 96) staged in K
  chunks of 16; or 128 threads (4 warps), up to four blocks per SM, the
  exact tile computed in two column passes with K chunks of 8, so that four
  instances' staging fits in the SM's shared memory.  More instances per SM
  hide more of the latency of each instance's chain of block-wide steps;
  fewer threads per instance make each step longer.
* ctas_per_sm: resident blocks per SM (the staging area is sized to fit
  them); more blocks also put more per-block workspace (about 15 n^2 doubles
  each) into L2.
* factor_smem: the Schur factorisation in shared memory (the whole m x m
  matrix loaded once, factored there, stored once) when the staging area
  holds it, or blocked from L2 with the GEMM tiles on the FP64 MMA.
* mixed_products (mixed precision only): the n^3 products of the FP32 phase
  on the FP64 MMA (0) or in FP32 on the SIMT pipe (1).

The tuner times every candidate on the batch itself (device events after a
warm-up, best of `reps`) and keeps the fastest per (nmax size class,
precision).
"""
from __future__ import annotations

_cache: dict = {}

SHAPES = (
    {"block_threads": 256, "ctas_per_sm": 2},
    {"block_threads": 256, "ctas_per_sm": 1},
    {"block_threads": 128, "ctas_per_sm": 4},
    {"block_threads": 128, "ctas_per_sm": 3},
)


def size_class(nmax: int) -> int:
    for c in (32, 64, 96, 128, 256, 512):
        if nmax <= c:
            return c
    return 1024


def label(shape: dict) -> str:
    return ",".join(f"{k}={v}" for k, v in sorted(shape.items()))


def tune(db, precision: int = 0, candidates=None, reps: int = 2, run=None, stream=None) -> dict:
    """Times one solve step for each candidate shape (dicts of DeviceBatch.solve
    keyword arguments; default SHAPES, then on the fastest the shared-memory
    Schur factorisation and, for mixed precision, FP32 products); returns {"best": shape, "ms": {label:
    ms}, "class": nmax class} and caches the choice.  `run(shape)` issues the
    step (default: db.solve with that shape) on `stream`."""
    import torch
    from . import _native as N
    s = stream if stream is not None else torch.cuda.current_stream()
    if run is None:
        run = lambda shape: db.solve(precision=precision, stream=s, **shape)
    key = (size_class(db.P.nmax), precision)
    res, shapes = {}, {}

    def time(shape):
        run(shape)
        torch.cuda.synchronize()
        best = 1e30
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(s)
            run(shape)
            e1.record(s)
            e1.synchronize()
            best = min(best, e0.elapsed_time(e1))
        res[label(shape)] = best
        shapes[label(shape)] = dict(shape)

    for shape in (candidates or SHAPES):
        time(shape)
    if candidates is None:
        top = dict(shapes[min(res, key=res.get)])
        time(dict(top, factor_smem=1))
        if precision == N.PREC_MIXED:
            top = dict(shapes[min(res, key=res.get)])
            time(dict(top, mixed_products=1))
    choice = shapes[min(res, key=res.get)]
    _cache[key] = choice
    return {"best": choice, "ms": res, "class": key[0]}


def choice(nmax: int, precision: int = 0, default: dict | None = None) -> dict:
    return _cache.get((size_class(nmax), precision), default or dict(SHAPES[0]))
