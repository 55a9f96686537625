"""Batched solves across the GPUs of one node: one process per GPU
(torch.distributed, NCCL on GPUs, gloo in the CPU tests), independent
instances sharded across ranks.

The instances of a batch never exchange data while they are solved, so the
only collective is one all-gather of the per-instance results at the end;
nothing crosses NVLink during the solve.  Instances are dealt to ranks by
estimated cost (n^3 + m^3 per iteration, largest first, each to the least
loaded rank), so ranks finish close together.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


def cost(n: int, m: int) -> float:
    """Per-iteration work estimate of one instance (Schur factor m^3/3 plus
    the O(n^3) block operations)."""
    return float(m) ** 3 / 3.0 + 14.0 * float(n) ** 3


def instance_size(it) -> tuple[int, int]:
    """(n, m) of an instance for cost(): the batched engine lays all its
    blocks (SDP and LP) along the diagonal of one matrix of order
    sum |size| and runs its dense steps on that whole matrix."""
    return int(sum(abs(int(b)) for b in it.blocks)), int(it.m)


def assign(sizes: list[tuple[int, int]], world: int) -> list[list[int]]:
    """Instance indices per rank: longest-processing-time-first dealing by
    cost(n, m).  Deterministic (ties broken by index), so every rank computes
    the same assignment without communicating."""
    order = sorted(range(len(sizes)), key=lambda q: (-cost(*sizes[q]), q))
    load = [0.0] * world
    out: list[list[int]] = [[] for _ in range(world)]
    for q in order:
        r = min(range(world), key=lambda k: (load[k], k))
        out[r].append(q)
        load[r] += cost(*sizes[q])
    for r in range(world):
        out[r].sort()
    return out


@dataclass
class ShardResult:
    """Per-instance results in the caller's instance order."""
    primal_obj: np.ndarray
    dual_obj: np.ndarray
    iterations: np.ndarray
    phase: np.ndarray
    status: np.ndarray
    x: list            # x (SDPA's xVec) per instance
    rank_of: np.ndarray  # which rank solved each instance


def solve_sharded(instances, solve_fn=None, group=None, **solve_kw) -> ShardResult:
    """Solves `instances` across the ranks of the default (or given) process
    group: each rank solves its share with `solve_fn(instances) -> (Packed,
    BatchResult)` (default: the batched CUDA solver through
    sdpab_batch_solve_host on this rank's current device), then the results
    are all-gathered so that every rank returns the whole batch."""
    import torch.distributed as dist
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    sizes = [instance_size(it) for it in instances]
    mine = assign(sizes, world)[rank]
    if solve_fn is None:
        from . import batch
        solve_fn = lambda its: (lambda P: (P, batch.solve_host(P, **solve_kw)))(batch.pack(its))
    part = {}
    if mine:
        P, r = solve_fn([instances[q] for q in mine])
        for t, q in enumerate(mine):
            part[q] = (float(r.primal_obj[t]), float(r.dual_obj[t]), int(r.iterations[t]), int(r.phase[t]),
                       int(r.status[t]), np.array(r.x_of(P, t)), rank)
    if world > 1:
        parts = [None] * world
        dist.all_gather_object(parts, part, group=group)
    else:
        parts = [part]
    merged = {}
    for p in parts:
        merged.update(p)
    if len(merged) != len(instances):
        raise RuntimeError(f"solve_sharded: gathered {len(merged)} of {len(instances)} results")
    cols = list(zip(*(merged[q] for q in range(len(instances)))))
    return ShardResult(np.array(cols[0]), np.array(cols[1]), np.array(cols[2], np.int32),
                       np.array(cols[3], np.int32), np.array(cols[4], np.int32), list(cols[5]),
                       np.array(cols[6], np.int32))
