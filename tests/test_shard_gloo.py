"""Multi-GPU path on CPU: sdpa_b200.shard deals independent instances to
ranks by cost and all-gathers the results; two gloo ranks (127.0.0.1) with
the oracle as the per-rank solver must return exactly the single-process
results, in the caller's order, on every rank."""
import os
import pickle
import socket

import numpy as np
import pytest


def _instances():
    from sdpa_b200 import instances as I
    return [I.batch_maxcut(s, 6, 14) for s in range(7)]


class _OracleBatch:
    """The oracle standing in for the GPU solver inside each rank."""

    def __init__(self, its):
        from oracle import sdpa_oracle as O
        rs = [O.solve(O.parse_dats(it.to_dats())) for it in its]
        self.primal_obj = np.array([r.primal_obj for r in rs])
        self.dual_obj = np.array([r.dual_obj for r in rs])
        self.iterations = np.array([r.iterations for r in rs])
        self.phase = np.array([r.phase for r in rs])
        self.status = np.zeros(len(rs), np.int32)
        self._x = [np.asarray(r.xvec) for r in rs]

    def x_of(self, P, t):
        return self._x[t]


def _worker(rank, world, port, out):
    import torch.distributed as dist
    from sdpa_b200 import shard
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        its = _instances()
        r = shard.solve_sharded(its, solve_fn=lambda sub: (None, _OracleBatch(sub)))
        with open(f"{out}.{rank}", "wb") as f:
            pickle.dump(r, f)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_assignment_balances_and_covers():
    from sdpa_b200 import shard
    sizes = [(n, n) for n in (120, 20, 80, 80, 40, 100, 60, 30)]
    a = shard.assign(sizes, 3)
    assert sorted(q for part in a for q in part) == list(range(len(sizes)))
    loads = [sum(shard.cost(*sizes[q]) for q in part) for part in a]
    assert max(loads) <= 1.35 * (sum(loads) / 3)
    assert shard.assign(sizes, 3) == a  # deterministic


def test_cost_counts_every_block():
    from sdpa_b200 import instances as I
    from sdpa_b200 import shard
    it = I.batch_block_sdp(3)
    n, m = shard.instance_size(it)
    assert n == sum(abs(int(b)) for b in it.blocks) and n > abs(int(it.blocks[0])) and m == it.m


def test_two_gloo_ranks_match_single_process(tmp_path):
    import torch.multiprocessing as mp
    from sdpa_b200 import shard
    out = str(tmp_path / "res")
    mp.spawn(_worker, args=(2, _free_port(), out), nprocs=2, join=True)
    single = shard.solve_sharded(_instances(), solve_fn=lambda sub: (None, _OracleBatch(sub)))
    for rank in range(2):
        with open(f"{out}.{rank}", "rb") as f:
            r = pickle.load(f)
        assert set(r.rank_of.tolist()) == {0, 1}
        np.testing.assert_array_equal(r.iterations, single.iterations)
        np.testing.assert_array_equal(r.primal_obj, single.primal_obj)
        for a, b in zip(r.x, single.x):
            np.testing.assert_array_equal(a, b)
