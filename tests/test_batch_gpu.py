"""Batched persistent solver (sdpab_batch_solve_host / sdpab_batch_solve)
against the reference solver's results (golden fixtures) and the oracle."""
import importlib.util
import os

import numpy as np
import pytest

from golden_util import GOLDEN, blocks, rel, small, tight, x_within_reference_accuracy

pytestmark = pytest.mark.gpu

_spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLDEN, "make_golden.py"))
MG = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(MG)

# Parity bar (floating point): objectives within 1e-6 relative of the
# reference, x within 1e-5 (absolute, as the values are O(1)..O(10)).
OBJ_TOL = 1e-6
X_TOL = 1e-5


def _solve(names, precision=0, **kw):
    from sdpa_b200 import batch
    cases = dict(MG.small_cases())
    insts = [cases[n] for n in names]
    P = batch.pack(insts)
    return P, batch.solve_host(P, precision=precision, **kw)


def test_batched_maxcut_matches_reference():
    meta, arr = small()
    names = [f"bmc{s}" for s in range(64)] + ["mc100", "mc20", "mc50w"]
    P, r = _solve(names, want_mats=True)
    iters_equal = 0
    for q, nm in enumerate(names):
        g = meta[nm]
        assert r.status[q] == 0
        assert r.phase[q] == 7, (nm, r.phase[q])  # pdOPT
        assert rel(r.primal_obj[q], g["primal_obj"]) < OBJ_TOL, nm
        assert rel(r.dual_obj[q], g["dual_obj"]) < OBJ_TOL, nm
        assert np.max(np.abs(r.x_of(P, q) - arr[nm + ".xvec"])) < X_TOL, nm
        iters_equal += int(r.iterations[q] == g["iterations"])
        assert abs(int(r.iterations[q]) - g["iterations"]) <= 1
    assert iters_equal >= len(names) - 2
    q = names.index("mc100")
    Y = r.mat_of(r.Y, P, q)
    assert np.max(np.abs(Y - arr["mc100.Y1"].reshape(100, 100, order="F"))) < 1e-4


def test_batched_general_constraints_match_reference():
    """Lovasz theta (m > n, two-entry constraints) through the same kernel."""
    meta, arr = small()
    names = ["lt20", "lt40"]
    P, r = _solve(names)
    for q, nm in enumerate(names):
        g = meta[nm]
        assert r.phase[q] == 7
        assert rel(r.primal_obj[q], g["primal_obj"]) < OBJ_TOL
        assert rel(r.dual_obj[q], g["dual_obj"]) < OBJ_TOL
        assert np.max(np.abs(r.x_of(P, q) - arr[nm + ".xvec"])) < X_TOL


def test_device_path_equals_host_path():
    import torch
    from sdpa_b200 import batch
    cases = dict(MG.small_cases())
    insts = [cases[f"bmc{s}"] for s in range(16)]
    P = batch.pack(insts)
    h = batch.solve_host(P)
    db = batch.DeviceBatch(P)
    db.solve()
    torch.cuda.synchronize()
    d = db.result()
    assert np.array_equal(h.iterations, d.iterations)
    assert np.allclose(h.primal_obj, d.primal_obj, rtol=1e-12, atol=0)


def test_empty_and_oversized_instances():
    from sdpa_b200 import batch, instances
    P = batch.pack([instances.batch_maxcut(3)])
    P.n[0] = 5000  # larger than the supported block order: rejected with a code
    with pytest.raises(Exception):
        batch.solve_host(P)


def test_batched_mixed_precision_matches_reference():
    """Mixed precision leaves the reference's iterate sequence: objectives
    within the parity tolerance, x at least as close to the reference's
    tight optimum as the reference's own x."""
    meta, arr = small()
    _, tz = tight()
    names = [f"bmc{s}" for s in range(64)] + ["mc100", "mc20", "mc50w", "lt20", "lt40"]
    P, r = _solve(names, precision=1)
    for q, nm in enumerate(names):
        g = meta[nm]
        assert r.phase[q] == 7, (nm, r.phase[q])
        assert rel(r.primal_obj[q], g["primal_obj"]) < OBJ_TOL, nm
        assert rel(r.dual_obj[q], g["dual_obj"]) < OBJ_TOL, nm
        assert x_within_reference_accuracy(r.x_of(P, q), arr[nm + ".xvec"], tz[nm + ".tight"]), nm


def _block_batch():
    """blk0..blk31, the small multi-block reference cases and two MaxCut
    instances in one batch."""
    from sdpa_b200 import batch
    bc = dict(MG.block_cases())
    sc = dict(MG.small_cases())
    names = [f"blk{s}" for s in range(32)] + ["rnd40", "rnd120", "ex2", "bmc0", "bmc1"]
    insts = [bc[n] if n.startswith("blk") else sc[n] for n in names]
    return names, insts, batch.pack(insts)


def _golden(nm):
    meta, arr = blocks() if nm.startswith("blk") else small()
    return meta[nm], arr


def test_batched_block_instances_match_reference():
    """Several SDP blocks and an LP block per instance (block-diagonal
    layout, per-block step length) against the reference's results."""
    from sdpa_b200 import batch
    names, insts, P = _block_batch()
    assert P.nblock is not None
    r = batch.solve_host(P, want_mats=True)
    iters_equal = 0
    for q, nm in enumerate(names):
        g, arr = _golden(nm)
        assert r.status[q] == 0, (nm, r.status[q])
        assert r.phase[q] == 7, (nm, r.phase[q])
        assert rel(r.primal_obj[q], g["primal_obj"]) < OBJ_TOL, nm
        assert rel(r.dual_obj[q], g["dual_obj"]) < OBJ_TOL, nm
        assert np.max(np.abs(r.x_of(P, q) - arr[nm + ".xvec"])) < X_TOL, nm
        iters_equal += int(r.iterations[q] == g["iterations"])
        assert abs(int(r.iterations[q]) - g["iterations"]) <= 1, nm
    assert iters_equal >= len(names) - 3
    # every block of X (getResultXMat) and Y (getResultYMat); off-block zero
    for q, nm in enumerate(names):
        if nm not in [f"blk{s}" for s in range(8)] + ["rnd40", "ex2"]:
            continue
        _, arr = _golden(nm)
        for l, b in enumerate(insts[q].blocks):
            for which, key in ((r.X, "X"), (r.Y, "Y")):
                ref = arr[f"{nm}.{key}{l + 1}"]
                got = r.block_of(which, P, q, l).ravel(order="F")
                assert np.max(np.abs(got - ref)) < 1e-4 * max(1.0, np.max(np.abs(ref))), (nm, key, l)
        M = r.mat_of(r.Y, P, q)
        mask = np.zeros(M.shape, bool)
        o = 0
        for b in insts[q].blocks:
            k = abs(b)
            if b > 0:
                mask[o:o + k, o:o + k] = True
            else:
                mask[np.arange(o, o + k), np.arange(o, o + k)] = True
            o += k
        assert np.all(M[~mask] == 0.0), nm


def test_block_device_path_equals_host_path():
    import torch
    from sdpa_b200 import batch
    names, insts, P = _block_batch()
    h = batch.solve_host(P)
    db = batch.DeviceBatch(P)
    db.solve()
    torch.cuda.synchronize()
    d = db.result()
    # Entries of several constraints at one position are summed into the
    # dense D and dZ by atomic adds, whose order varies between runs: equal
    # iteration counts, objectives equal to rounding.
    assert np.array_equal(h.iterations, d.iterations)
    assert np.allclose(h.primal_obj, d.primal_obj, rtol=1e-9, atol=0)


def test_block_warm_start_uses_diagonal_blocks_only():
    """SDPAB_INIT_POINT on block instances: a point near the reference's
    solution whose off-block entries are garbage; the solver keeps the
    diagonal blocks only, starts there and reaches the reference's optimum."""
    from sdpa_b200 import batch
    names, insts, P = _block_batch()
    sel = [q for q, nm in enumerate(names) if nm in [f"blk{s}" for s in range(8)]]
    its = [insts[q] for q in sel]
    P = batch.pack(its)
    X = np.zeros(P.nden)
    Y = np.zeros(P.nden)
    xv = np.zeros(P.nvec)
    for q, nm in enumerate([names[i] for i in sel]):
        _, arr = _golden(nm)
        n = int(P.n[q])
        Xq = np.full((n, n), 0.37)
        Yq = np.full((n, n), -0.21)
        o = 0
        for l, b in enumerate(its[q].blocks):
            k = abs(b)
            for M, key in ((Xq, "X"), (Yq, "Y")):
                ref = arr[f"{nm}.{key}{l + 1}"]
                blk = np.diag(ref) if b < 0 else ref.reshape(k, k, order="F")
                M[o:o + k, o:o + k] = 0.9 * blk + 0.1 * np.eye(k)
            o += k
        X[P.dense_off[q]:P.dense_off[q] + n * n] = Xq.ravel(order="F")
        Y[P.dense_off[q]:P.dense_off[q] + n * n] = Yq.ravel(order="F")
        xv[P.vec_off[q]:P.vec_off[q] + P.m[q]] = arr[nm + ".xvec"]
    flag = np.full(P.count, 1, np.int32)
    r = batch.solve_host(P, init=(flag, xv, X, Y))
    for q, nm in enumerate([names[i] for i in sel]):
        g, _ = _golden(nm)
        assert r.status[q] in (0, 2), (nm, r.status[q])
        assert r.phase[q] == 7, nm
        assert rel(r.primal_obj[q], g["primal_obj"]) < OBJ_TOL, nm
        assert rel(r.dual_obj[q], g["dual_obj"]) < OBJ_TOL, nm
    assert int(np.sum(r.status == 0)) >= len(sel) // 2


def test_batched_dense_constraints_single_block_match_reference():
    """The general solver on one SDP block with dense constraints (F1 columns
    with a full-order product, no block structure to exploit)."""
    from sdpa_b200 import batch
    meta, arr = blocks()
    cases = MG.dense_cases()
    P = batch.pack([it for _, it in cases])
    r = batch.solve_host(P, want_mats=True)
    for q, (nm, it) in enumerate(cases):
        g = meta[nm]
        assert r.status[q] == 0 and r.phase[q] == 7, (nm, r.status[q], r.phase[q])
        assert rel(r.primal_obj[q], g["primal_obj"]) < OBJ_TOL, nm
        assert rel(r.dual_obj[q], g["dual_obj"]) < OBJ_TOL, nm
        assert np.max(np.abs(r.x_of(P, q) - arr[nm + ".xvec"])) < X_TOL, nm
        assert abs(int(r.iterations[q]) - g["iterations"]) <= 1, nm
        Y = r.block_of(r.Y, P, q, 0).ravel(order="F")
        ref = arr[nm + ".Y1"]
        assert np.max(np.abs(Y - ref)) < 1e-4 * max(1.0, np.max(np.abs(ref))), nm


@pytest.mark.parametrize("shape", [{"block_threads": 128, "ctas_per_sm": 4}, {"block_threads": 128, "ctas_per_sm": 3},
                                   {"block_threads": 256, "ctas_per_sm": 1}, {"factor_smem": 1},
                                   {"factor_smem": 1, "block_threads": 128}])
def test_launch_shapes_match_reference(shape):
    """Every launch shape the autotuner may pick (128-thread blocks, whose
    products run as two-pass exact tiles with K chunks of 8; fewer
    256-thread blocks per SM; the Schur factorisation in shared memory)
    solves to the same results: FP64 single-block
    and multi-block batches against the reference (strict bar), and mixed
    precision with either product precision (reference-accuracy bar)."""
    from sdpa_b200 import batch
    meta, arr = small()
    _, tz = tight()
    names = [f"bmc{s}" for s in range(64)] + ["mc100", "mc20", "mc50w"]
    P, r = _solve(names, **shape)
    for q, nm in enumerate(names):
        g = meta[nm]
        assert r.status[q] == 0 and r.phase[q] == 7, (nm, r.phase[q])
        assert rel(r.primal_obj[q], g["primal_obj"]) < OBJ_TOL, nm
        assert np.max(np.abs(r.x_of(P, q) - arr[nm + ".xvec"])) < X_TOL, nm
        assert abs(int(r.iterations[q]) - g["iterations"]) <= 1
    bnames, insts, BP = _block_batch()
    rb = batch.solve_host(BP, **shape)
    for q, nm in enumerate(bnames):
        g, garr = _golden(nm)
        assert rb.status[q] == 0 and rb.phase[q] == 7, (nm, rb.status[q], rb.phase[q])
        assert rel(rb.primal_obj[q], g["primal_obj"]) < OBJ_TOL, nm
        assert np.max(np.abs(rb.x_of(BP, q) - garr[nm + ".xvec"])) < X_TOL, nm
    mnames = names + ["lt20", "lt40"]
    for mp in (0, 1):
        P2, r2 = _solve(mnames, precision=1, mixed_products=mp, **shape)
        for q, nm in enumerate(mnames):
            g = meta[nm]
            assert r2.phase[q] == 7, (nm, mp, r2.phase[q])
            assert rel(r2.primal_obj[q], g["primal_obj"]) < OBJ_TOL, (nm, mp)
            assert rel(r2.dual_obj[q], g["dual_obj"]) < OBJ_TOL, (nm, mp)
            assert x_within_reference_accuracy(r2.x_of(P2, q), arr[nm + ".xvec"], tz[nm + ".tight"]), (nm, mp)


def test_mixed_precision_refines_in_fp32_phase():
    """Mixed precision with the FP32 Schur factor and FP64 refinement over a
    wide FP32 phase (switch at relative gap 1e-5): the solve still reaches
    pdOPT with the reference's objectives on every instance."""
    meta, arr = small()
    _, tz = tight()
    names = [f"bmc{s}" for s in range(64)]
    P, r = _solve(names, precision=1, mixed_switch_gap=1e-5)
    for q, nm in enumerate(names):
        g = meta[nm]
        assert r.phase[q] == 7, (nm, r.phase[q])
        assert rel(r.primal_obj[q], g["primal_obj"]) < OBJ_TOL, nm
        assert rel(r.dual_obj[q], g["dual_obj"]) < OBJ_TOL, nm
