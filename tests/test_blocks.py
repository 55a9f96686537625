"""Multi-block batches on the CPU: the oracle against the reference's
results on the batched multi-block family (several SDP blocks and an LP
block), the packed layout of sdpab_batch's block structure, and the host
entry point's rejection of malformed structures (before any device call)."""
import importlib.util
import os

import numpy as np
import pytest

from golden_util import GOLDEN, blocks, rel
from oracle import sdpa_oracle as O

_spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLDEN, "make_golden.py"))
MG = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(MG)


def test_oracle_matches_reference_on_block_instances():
    meta, arr = blocks()
    cases = dict(MG.block_cases())
    for name in ("blk0", "blk2", "blk3", "blk5"):
        r = O.solve(O.parse_dats(cases[name].to_dats()))
        g = meta[name]
        assert O.PHASE_NAMES[r.phase] == g["phase"] == "pdOPT"
        assert r.iterations == g["iterations"], name
        assert rel(r.primal_obj, g["primal_obj"]) < 1e-8, name
        assert rel(r.dual_obj, g["dual_obj"]) < 1e-8, name
        assert np.max(np.abs(r.xvec - arr[name + ".xvec"])) < 1e-6, name


def test_block_family_shapes():
    from sdpa_b200 import instances
    for s in range(32):
        it = instances.batch_block_sdp(s)
        sdp = [b for b in it.blocks if b > 0]
        assert 2 <= len(sdp) <= 4 and all(6 <= b <= 40 for b in sdp)
        assert all(-12 <= b < 0 for b in it.blocks if b < 0)
        assert 10 <= it.m <= 80
        # entries inside their block, LP entries diagonal
        sz = np.abs(np.asarray(it.blocks))[it.l - 1]
        assert np.all((it.i >= 1) & (it.j <= sz) & (it.i <= it.j))
        lp = np.asarray(it.blocks)[it.l - 1] < 0
        assert np.all(it.i[lp] == it.j[lp])


def test_pack_lays_blocks_along_the_diagonal():
    from sdpa_b200 import batch, instances
    its = [instances.batch_block_sdp(2), instances.batch_maxcut(1)]
    P = batch.pack(its)
    assert P.nblock is not None and list(P.nblock) == [len(its[0].blocks), 1]
    assert P.blocks_of(0) == its[0].blocks and P.blocks_of(1) == [its[1].m]
    assert P.n[0] == sum(abs(b) for b in its[0].blocks)
    offs = np.concatenate([[0], np.cumsum(np.abs(its[0].blocks))])
    # every entry of instance 0 maps to its block's rows and columns
    e0, e1 = P.mat_ptr[P.mat_off[0]], P.mat_ptr[P.mat_off[0] + its[0].m + 1]
    r, c = P.row[e0:e1], P.col[e0:e1]
    blk_r = np.searchsorted(offs, r, side="right") - 1
    blk_c = np.searchsorted(offs, c, side="right") - 1
    assert np.array_equal(blk_r, blk_c)
    lp = np.asarray(its[0].blocks)[blk_r] < 0
    assert np.all(r[lp] == c[lp])
    # a batch of single SDP blocks carries no block structure
    assert batch.pack([instances.batch_maxcut(s) for s in range(3)]).nblock is None


@pytest.mark.parametrize("mutate", ["sum", "zero", "count"])
def test_host_entry_rejects_malformed_structure(mutate):
    from sdpa_b200 import _native as N
    from sdpa_b200 import batch, instances
    P = batch.pack([instances.batch_block_sdp(1)])
    if mutate == "sum":
        P.blk_size = P.blk_size.copy()
        P.blk_size[0] += 1      # orders no longer add up to n
    elif mutate == "zero":
        P.blk_size = P.blk_size.copy()
        P.blk_size[-1] = 0      # a block of order 0
    else:
        P.nblock = np.array([N.BATCH_MAX_BLOCKS + 1], np.int32)
    with pytest.raises(N.SolverError, match="nblock|order|add up"):
        batch.solve_host(P)


def test_dense_constraint_instances_take_the_general_solver():
    """Single-block instances whose constraints have more than 2n effective
    entries carry a block structure, which selects the solver with F1
    columns; the oracle matches the reference on two of them."""
    from sdpa_b200 import batch
    meta, arr = blocks()
    cases = MG.dense_cases()
    P = batch.pack([it for _, it in cases])
    assert P.nblock is not None and all(P.blocks_of(q) == it.blocks for q, (_, it) in enumerate(cases))
    for name, it in cases[:2]:
        r = O.solve(O.parse_dats(it.to_dats()))
        g = meta[name]
        assert r.iterations == g["iterations"], name
        assert rel(r.primal_obj, g["primal_obj"]) < 1e-8, name
        assert np.max(np.abs(r.xvec - arr[name + ".xvec"])) < 1e-6, name


def test_block_arrow_family_and_its_fixture():
    """The block-arrow family: separable constraints grouped by block, then
    coupling constraints on two blocks each; its fixture comes from the
    numpy restatement (the reference itself needs MUMPS for it)."""
    import json
    from sdpa_b200 import instances
    it = instances.block_arrow_sdp()
    assert it.m == 24 * 24 + 8 and it.blocks == [8] * 24
    blk_of = {}
    for k, l in zip(it.k, it.l):
        if k > 0:
            blk_of.setdefault(int(k), set()).add(int(l))
    assert all(blk_of[k] == {(k - 1) // 24 + 1} for k in range(1, 24 * 24 + 1))
    assert all(len(blk_of[k]) == 2 for k in range(24 * 24 + 1, it.m + 1))
    meta = json.load(open(os.path.join(GOLDEN, "arrow.json")))["arrow"]
    assert meta["phase"] == "pdOPT" and "restatement" in meta["source"]


def _constraint_order(inst):
    import ctypes
    from sdpa_b200 import _native as N
    m = inst.m
    bs = np.asarray(inst.blocks, np.int32)
    k, l, i, j = [np.ascontiguousarray(a, np.int32) for a in (inst.k, inst.l, inst.i, inst.j)]
    out = np.zeros(m, np.int32)
    pairs = np.zeros(2, np.int64)
    rc = N.lib().sdpab_constraint_order(m, len(bs), bs.ctypes.data, len(k), k.ctypes.data, l.ctypes.data,
                                        i.ctypes.data, j.ctypes.data, out.ctypes.data, pairs.ctypes.data)
    assert rc == 0
    return out, pairs


def test_constraint_order_restores_the_arrowhead():
    """The host solver's constraint order for the Schur factorisation (host
    code, no device): a block-arrow problem whose constraints come in a
    shuffled order has a dense symbolic tile pattern in that order; the
    chosen order (the fewest tile pairs among minimum degree, the
    group-count order and the caller's) is a permutation that brings back
    the arrowhead: constraints local to one block contiguous, the coupling
    ones last, and as few tile pairs as the problem in its generated order.
    A single-block problem keeps the caller's order."""
    from sdpa_b200 import instances
    grouped = instances.block_arrow_sdp(nblk=200, m_per=40, n_couple=64)
    shuffled = instances.block_arrow_sdp(nblk=200, m_per=40, n_couple=64, shuffled=True)
    o_g, p_g = _constraint_order(grouped)
    o_s, p_s = _constraint_order(shuffled)
    assert sorted(o_s.tolist()) == list(range(shuffled.m))
    assert p_s[0] > 10 * p_s[1], p_s
    assert p_s[1] <= p_g[1] and p_g[1] <= p_g[0]
    # which block each constraint touches (the coupling ones: two)
    blocks_of = [set() for _ in range(shuffled.m)]
    for kk, ll in zip(shuffled.k, shuffled.l):
        if kk > 0:
            blocks_of[kk - 1].add(int(ll))
    seq = [blocks_of[c] for c in o_s]
    n_local = sum(1 for b in seq if len(b) == 1)
    assert all(len(b) == 1 for b in seq[:n_local]) and all(len(b) == 2 for b in seq[n_local:])
    firsts = [min(b) for b in seq[:n_local]]
    changes = sum(1 for a, b in zip(firsts, firsts[1:]) if a != b)
    assert changes == 199  # each block's constraints contiguous
    lt = instances.lovasz_theta(n=60, p=0.5, seed=1)
    o_lt, p_lt = _constraint_order(lt)
    assert np.array_equal(o_lt, np.arange(lt.m)) and p_lt[0] == p_lt[1]
