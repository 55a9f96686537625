"""The low-rank factor start (sdpab_lowrank_factor + SDPAB_INIT_FACTOR).

* The mixing-method kernel against a numpy restatement of the same
  iteration (same seeded start, rows in the kernel's colour order): Y = V V^T
  agrees after a fixed number of sweeps.
* The benchmark's headline set (first 512 instances of the 4096-instance
  MaxCut batch) solved from the factor start against the reference SDPA's
  own results (tests/golden/headline.*): every instance pdOPT with both
  objectives within 1e-6; x within 1e-5 of the reference's or no farther
  from its epsilonStar = 1e-11 solution than the reference's own x (the
  bar of oracle.ref_runner.x_within_reference_accuracy) for all but 2 %;
  the median and 99th percentile of the distance to that solution no larger
  than the reference's, the largest within 1.5 times the reference's; at
  most 1 % of the instances solved again from the standard start (status
  2); and the iterations cut to at most 4 on average (the reference takes
  about 14).
* Instances not of the form X_ii = b_i are reported (-1 sweeps) and solved
  from the standard start, and the host-pointer entry point takes the same
  start.
"""
import json
import os

import numpy as np
import pytest

from golden_util import GOLDEN

pytestmark = pytest.mark.gpu

SEEDS = 512
M64 = (1 << 64) - 1


def _uniform(seed, q, i, k):
    """splitmix64 of the kernel's per-entry counter, mapped to [-1, 1)."""
    ctr = (q * 65536 * 64 + i * 64 + k + 1) & M64
    z = (seed + 0x9E3779B97F4A7C15 * ctr) & M64
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
    z ^= z >> 31
    return (z >> 11) * (2.0 / 9007199254740992.0) - 1.0


def _f0(it, n):
    F0 = np.zeros((n, n))
    for k, i, j, v in zip(it.k, it.i, it.j, it.v):
        if k == 0:
            F0[i - 1, j - 1] = v
            F0[j - 1, i - 1] = v
    return F0


def _update_order(A):
    """The kernel's row order: greedy colours in row order (the smallest
    colour below 64 no earlier neighbour has, else a class of its own after
    all others), rows by colour, in row order within a colour."""
    n = A.shape[0]
    col = np.full(n, -1)
    for i in range(n):
        used = {int(col[j]) for j in np.nonzero(A[i])[0] if 0 <= col[j] < 64}
        free = [c for c in range(64) if c not in used]
        col[i] = free[0] if free else 64 + i
    return sorted(range(n), key=lambda i: (min(col[i], 64), i))


def _mixing(F0, rq, R, seed, q, sweeps):
    n = F0.shape[0]
    V = np.zeros((n, R))
    for i in range(n):
        V[i, :rq] = [_uniform(seed, q, i, k) for k in range(rq)]
        V[i] /= np.linalg.norm(V[i])
    A = F0 - np.diag(np.diag(F0))
    order = _update_order(A)
    for _ in range(sweeps):
        for i in order:
            g = A[i] @ V
            nr = np.linalg.norm(g)
            if nr > 0:
                V[i] = g / nr
    return V


def test_factor_matches_numpy_restatement():
    import math
    import torch
    from sdpa_b200 import batch, instances, lowrank
    seeds = [0, 3, 11, 23]
    its = [instances.batch_maxcut(s, 20, 120) for s in seeds]
    P = batch.pack(its)
    db = batch.DeviceBatch(P)
    fp = lowrank.FactorPipeline(db, max_sweeps=25, tol=0.0, seed=7)
    fp.factor()
    torch.cuda.synchronize()
    V = fp.V.cpu().numpy()
    assert np.all(fp.sweeps.cpu().numpy() == 25)
    for q, it in enumerate(its):
        n = it.blocks[0]
        rq = min(fp.rank, int(math.ceil(math.sqrt(2 * n))) + 1)
        Vg = V[P.vec_off[q] * fp.rank:(P.vec_off[q] + n) * fp.rank].reshape(n, fp.rank)
        Vn = _mixing(_f0(it, n), rq, fp.rank, 7, q, 25)
        assert np.all(Vg[:, rq:] == 0.0)
        assert np.max(np.abs(Vg @ Vg.T - Vn @ Vn.T)) < 1e-9


def test_factor_start_matches_reference():
    import torch
    from oracle.ref_runner import x_within_reference_accuracy
    from sdpa_b200 import batch, instances, lowrank
    meta = json.load(open(os.path.join(GOLDEN, "headline.json")))
    arr = np.load(os.path.join(GOLDEN, "headline.npz"))
    P = batch.pack([instances.batch_maxcut(s, 20, 120) for s in range(SEEDS)])
    db = batch.DeviceBatch(P)
    fp = lowrank.FactorPipeline(db)
    fp.run()
    torch.cuda.synchronize()
    res = db.result()
    rel = lambda a, b: abs(a - b) / max(1.0, abs(b))
    obj_bad, x_bad, e_ours, e_ref = [], [], [], []
    for q in range(SEEDS):
        if (res.phase[q] != 7 or rel(res.primal_obj[q], meta["primal_obj"][q]) > 1e-6
                or rel(res.dual_obj[q], meta["dual_obj"][q]) > 1e-6):
            obj_bad.append(q)
        x, xr, xt = res.x_of(P, q), arr[f"bmc{q}.xvec"], arr[f"bmc{q}.tight"]
        e_ours.append(float(np.max(np.abs(x - xt))))
        e_ref.append(float(np.max(np.abs(xr - xt))))
        if not (np.max(np.abs(x - xr)) <= 1e-5 or x_within_reference_accuracy(x, xr, xt)):
            x_bad.append(q)
    e_ours, e_ref = np.array(e_ours), np.array(e_ref)
    print(f"factor start vs reference ({SEEDS}): objectives off {len(obj_bad)}, x outside both bars "
          f"{len(x_bad)}; |x - x*| median {np.median(e_ours):.2e} max {e_ours.max():.2e} (reference "
          f"{np.median(e_ref):.2e} / {e_ref.max():.2e}); iterations {res.iterations.mean():.2f}; sweeps "
          f"{fp.sweeps.float().mean().item():.1f}")
    assert not obj_bad, f"objective or phase differs from the reference: instances {obj_bad[:10]}"
    # a start from a factor that did not converge may stall; the solver then
    # solves that instance again from the standard start (status 2)
    assert np.all((res.status == 0) | (res.status == 2)) and np.sum(res.status == 2) <= 0.01 * SEEDS
    assert len(x_bad) <= 0.02 * SEEDS, f"x outside both bars: instances {x_bad[:10]}"
    # the stopping test (relative gap 1e-7) leaves x undetermined to about
    # 1e-4 on the worst instances, for the reference as here: the tail is
    # compared with a margin, the bulk strictly
    assert np.median(e_ours) <= np.median(e_ref)
    assert np.percentile(e_ours, 99) <= np.percentile(e_ref, 99) and e_ours.max() <= 1.5 * e_ref.max()
    assert res.iterations.mean() <= 4.0


def test_factor_start_other_forms_and_host_entry():
    import torch
    from sdpa_b200 import batch, instances, lowrank
    its = [instances.batch_maxcut(5, 20, 60), instances.random_sdp(m=30, n=12, nlp=4, density=0.3, seed=2),
           instances.batch_maxcut(6, 20, 60)]
    P = batch.pack(its)
    db = batch.DeviceBatch(P)
    fp = lowrank.FactorPipeline(db)
    fp.run()
    torch.cuda.synchronize()
    res = db.result()
    sw = fp.sweeps.cpu().numpy()
    assert sw[1] == -1 and sw[0] > 0 and sw[2] > 0
    assert list(res.status) == [0, 1, 0]
    assert np.all(res.phase == 7)
    cold = batch.solve_host(P)
    assert abs(res.primal_obj[1] - cold.primal_obj[1]) <= 1e-6 * max(1.0, abs(cold.primal_obj[1]))
    # the host-pointer entry point from the same factors: the same solve
    flag = np.full(P.count, lowrank.INIT_FACTOR, np.int32)
    hres = batch.solve_host(P, init=(flag, None, None, None, 0.0, fp.V.cpu().numpy(), fp.rank))
    assert np.array_equal(hres.iterations, res.iterations)
    assert np.max(np.abs(hres.primal_obj - res.primal_obj) / np.maximum(1.0, np.abs(res.primal_obj))) < 1e-12
    assert np.max(np.abs(hres.xvec - res.xvec)) < 1e-9


def test_subsets_solve_like_the_whole_batch():
    """The factor and the solve of a batch in two instance subsets, on two
    streams for the factor (each call has its own work-queue counter), give
    the results of one call over the whole batch: the factors bitwise, the
    solves to rounding (every instance is computed on its own)."""
    import torch
    from sdpa_b200 import batch, instances, lowrank
    P = batch.pack([instances.batch_maxcut(s, 20, 120) for s in range(64)])
    dbw = batch.DeviceBatch(P)
    fw = lowrank.FactorPipeline(dbw)
    fw.run()
    dbs = batch.DeviceBatch(P)
    fs = lowrank.FactorPipeline(dbs)
    o = fs.order.cpu().numpy()
    a = torch.from_numpy(np.ascontiguousarray(o[::2])).cuda()
    b = torch.from_numpy(np.ascontiguousarray(o[1::2])).cuda()
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    fs.factor(side, a)
    fs.factor(None, b)
    torch.cuda.current_stream().wait_stream(side)
    dbs.solve(order=b)
    dbs.solve(order=a)
    torch.cuda.synchronize()
    assert torch.equal(fw.V, fs.V) and torch.equal(fw.sweeps, fs.sweeps)
    # the solver's shared-memory accumulations may add in another order from
    # one launch to the next: the same iterations, values to rounding
    rw, rs = dbw.result(), dbs.result()
    assert np.array_equal(rw.iterations, rs.iterations)
    assert np.max(np.abs(rw.primal_obj - rs.primal_obj) / np.maximum(1.0, np.abs(rw.primal_obj))) < 1e-12
    assert np.max(np.abs(rw.xvec - rs.xvec)) < 1e-9
