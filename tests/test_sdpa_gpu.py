"""The drop-in SDPA class (host-driven CUDA solver) through the whole-problem
C ABI, against the reference manual's known answers and the reference
solver's results (golden fixtures): multiple SDP blocks, LP blocks, F1 and
F3 Schur formulas, the .dat-s and .dat readers, warm start."""
import importlib.util
import os

import numpy as np
import pytest

from golden_util import GOLDEN, known_answers, large, rel, small, tight, x_within_reference_accuracy

pytestmark = pytest.mark.gpu

_spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLDEN, "make_golden.py"))
MG = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(MG)

OBJ_TOL = 1e-6   # relative objective tolerance
X_TOL = 1e-5     # absolute tolerance on x (SDPA's xVec)


def _solve(inst, params=None, path=None, sparse_type=0):
    from sdpa_b200.sdpa import SDPA
    s = SDPA()
    if params:
        s.setParameter(**params)
    if path:
        s.readInput(path, sparse_type)
    else:
        s.inputProblem(inst)
    s.solve()
    return s


def test_manual_examples():
    ka = known_answers()
    for name, inst in (("example1", MG.example1()), ("example2", MG.example2())):
        s = _solve(inst)
        man = ka["manual"][name]
        assert s.getPhaseString() == "pdOPT"
        assert s.getIteration() == man["iterations"], name
        assert rel(s.getPrimalObj(), man["primal_obj"]) < 1e-8
        assert rel(s.getDualObj(), man["dual_obj"]) < 1e-8
        ref = ka["reference_default"][name]
        assert np.max(np.abs(s.getResultXVec() - np.array(ref["xvec"]))) < X_TOL


def test_param_1e8_examples():
    ka = known_answers()
    prm = dict(maxIteration=200, epsilonStar=1e-8, lowerBound=-1e20, upperBound=1e20, epsilonDash=1e-8)
    for name, inst in (("example1", MG.example1()), ("example2", MG.example2())):
        s = _solve(inst, prm)
        ref = ka["reference_param_1e-8"][name]
        assert s.getIteration() == ref["iterations"]
        assert rel(s.getPrimalObj(), ref["primal_obj"]) < 1e-9


@pytest.mark.parametrize("name", ["mc100", "mc20", "mc50w", "lt20", "lt40", "rnd40", "rnd120", "ex2"])
def test_small_instances_match_reference(name, tmp_path):
    meta, arr = small()
    inst = dict(MG.small_cases())[name]
    path = str(tmp_path / f"{name}.dat-s")
    inst.write(path)
    s = _solve(None, path=path)   # through the .dat-s reader
    g = meta[name]
    assert s.getPhaseString() == g["phase"]
    assert abs(s.getIteration() - g["iterations"]) <= 1
    assert rel(s.getPrimalObj(), g["primal_obj"]) < OBJ_TOL
    assert rel(s.getDualObj(), g["dual_obj"]) < OBJ_TOL
    assert np.max(np.abs(s.getResultXVec() - arr[name + ".xvec"])) < X_TOL
    if name + ".Y1" in arr:
        Y = s.getResultYMat(1)
        assert np.max(np.abs(Y.ravel(order="F") - arr[name + ".Y1"])) < 1e-4


def test_dense_dat_reader(tmp_path):
    """example2 written in the dense .dat format (F0..Fm as full block matrices)."""
    ka = known_answers()
    inst = MG.example2()
    lines = ["*dense example2", "5", "3", "2 3 -2", " ".join(map(str, inst.c))]
    for k in range(6):
        B1, B2, lp = np.zeros((2, 2)), np.zeros((3, 3)), np.zeros(2)
        for kk, l, i, j, v in zip(inst.k, inst.l, inst.i, inst.j, inst.v):
            if kk != k:
                continue
            if l == 1:
                B1[i - 1, j - 1] = B1[j - 1, i - 1] = v
            elif l == 2:
                B2[i - 1, j - 1] = B2[j - 1, i - 1] = v
            else:
                lp[i - 1] = v
        lines.append("{ " + str(B1.tolist()) + str(B2.tolist()) + str(lp.tolist()) + " }")
    p = tmp_path / "example2.dat"
    p.write_text("\n".join(lines).replace("[", "{").replace("]", "}") + "\n")
    s = _solve(None, path=str(p))
    assert s.getIteration() == ka["manual"]["example2"]["iterations"]
    assert rel(s.getPrimalObj(), ka["manual"]["example2"]["primal_obj"]) < 1e-8


def test_warm_start_and_fallback():
    """copyCurrentToInit re-solve (example4 of the reference's libexample) and
    the strict-interiority fallback of a non-interior initial point."""
    from sdpa_b200.sdpa import SDPA
    inst = dict(MG.small_cases())["mc20"]
    s = SDPA()
    s.inputProblem(inst)
    s.solve()
    obj = s.getPrimalObj()
    x = s.getResultXVec()
    Xm, Ym = s.getResultXMat(1), s.getResultYMat(1)
    # a strictly interior point near the optimum: shift toward the centre
    t = SDPA()
    t.inputProblem(inst)
    t.setInitPoint(x - 0.1, [Xm + 0.1 * np.eye(20)], [0.9 * Ym + 0.1 * np.eye(20)])
    t.solve()
    assert t.getPhaseString() == "pdOPT"
    assert rel(t.getPrimalObj(), obj) < OBJ_TOL
    # a non-interior point (X indefinite) falls back to the standard start
    u = SDPA()
    u.inputProblem(inst)
    u.setInitPoint(np.zeros(20), [-np.eye(20)], [np.eye(20)])
    u.solve()
    assert u.getPhaseString() == "pdOPT"
    assert rel(u.getPrimalObj(), obj) < OBJ_TOL
    assert u.getIteration() == s.getIteration()


def test_dimacs_errors_small():
    s = _solve(MG.example1())
    d = s.getDimacsError()
    assert d[1] < 1e-7 and d[3] < 1e-7 and abs(d[5]) < 1e-6 and d[2] == 0.0 and d[4] == 0.0


@pytest.mark.parametrize("n", [1, 2, 3, 20, 21, 64, 200, 501])
def test_min_eigenvalue_matches_dense_solver(n):
    """sdpab_min_eigenvalue (the dsyev minimum of Lal::getMinEigenValue that
    the DIMACS errors take, computed on the GPU) against numpy's eigvalsh, on
    random symmetric matrices and on a positive semidefinite one of rank
    n - 1 (smallest eigenvalue 0)."""
    import ctypes
    import torch
    from sdpa_b200 import _native as N
    rng = np.random.default_rng(n)
    G = rng.standard_normal((n, n))
    V = rng.standard_normal((n, max(n - 1, 1)))
    for A in (0.5 * (G + G.T), V @ V.T if n > 1 else np.zeros((1, 1))):
        ref = np.linalg.eigvalsh(A)[0]
        # only the lower triangle is referenced: spoil the strict upper one
        Ad = np.tril(A) + np.triu(np.full((n, n), 7.0), 1)
        dev = torch.from_numpy(np.asfortranarray(Ad).ravel(order="F").copy()).cuda()
        out = ctypes.c_double()
        N.check(N.lib().sdpab_min_eigenvalue(n, dev.data_ptr(), ctypes.byref(out), None), "min_eigenvalue")
        scale = max(1.0, np.abs(np.linalg.eigvalsh(A)).max())
        assert abs(out.value - ref) <= 1e-12 * scale, (n, out.value, ref)


@pytest.mark.parametrize("name", ["lt200", "rnd2000"])
def test_large_configs_match_reference(name):
    """Lovasz theta G(200, 0.5) (m = 9986, F3, dense 9986^2 Schur) and the random
    m = 2000 SDP with blocks {500, LP 50} (F1 formula)."""
    from sdpa_b200 import instances
    meta, arr = large()
    if meta is None:
        pytest.skip("large fixtures not generated")
    inst = instances.lovasz_theta(200, 0.5, 1) if name == "lt200" else instances.random_sdp(seed=1)
    s = _solve(inst)
    g = meta[name]
    assert s.getPhaseString() == g["phase"]
    assert abs(s.getIteration() - g["iterations"]) <= 1
    assert rel(s.getPrimalObj(), g["primal_obj"]) < OBJ_TOL
    assert rel(s.getDualObj(), g["dual_obj"]) < OBJ_TOL
    assert np.max(np.abs(s.getResultXVec() - arr[name + ".xvec"])) < X_TOL


@pytest.mark.parametrize("name", ["mc100", "lt40", "rnd120", "ex2"])
def test_mixed_precision_small(name):
    """FP32 products / FP32 Schur factor + FP64 refinement (mixed) reach the
    same optimum as the reference within the parity tolerance."""
    from sdpa_b200.sdpa import SDPA
    meta, arr = small()
    inst = dict(MG.small_cases())[name]
    s = SDPA()
    s.setPrecision(1)
    s.inputProblem(inst)
    s.solve()
    g = meta[name]
    assert s.getPhaseString() == "pdOPT"
    assert rel(s.getPrimalObj(), g["primal_obj"]) < OBJ_TOL
    assert rel(s.getDualObj(), g["dual_obj"]) < OBJ_TOL
    _, tz = tight()
    assert x_within_reference_accuracy(s.getResultXVec(), arr[name + ".xvec"], tz[name + ".tight"])


@pytest.mark.parametrize("name", ["lt200", "rnd2000"])
def test_mixed_precision_large(name):
    from sdpa_b200 import instances
    from sdpa_b200.sdpa import SDPA
    meta, arr = large()
    if meta is None:
        pytest.skip("large fixtures not generated")
    inst = instances.lovasz_theta(200, 0.5, 1) if name == "lt200" else instances.random_sdp(seed=1)
    s = SDPA()
    s.setPrecision(1)
    s.inputProblem(inst)
    s.solve()
    g = meta[name]
    assert s.getPhaseString() == "pdOPT"
    assert rel(s.getPrimalObj(), g["primal_obj"]) < OBJ_TOL
    assert rel(s.getDualObj(), g["dual_obj"]) < OBJ_TOL
    x = s.getResultXVec()
    if name + ".tight" in arr.files:
        assert x_within_reference_accuracy(x, arr[name + ".xvec"], arr[name + ".tight"])
    else:  # no tight solution stored: the reference's x itself
        assert np.max(np.abs(x - arr[name + ".xvec"])) < X_TOL


def test_sparse_schur_on_a_block_arrow_problem(monkeypatch):
    """Many SDP blocks whose Schur matrix is block-diagonal with a dense
    border: the reference takes its sparse (MUMPS) Schur path here; this
    solver skips the 128 x 128 tiles of the factor its symbolic pattern
    leaves zero.  The automatic choice is the sparse path, the result
    matches the numpy restatement of the reference's algorithm, and the
    dense factorisation (SDPAB_SCHUR=dense) gives the same iterates to
    rounding."""
    import json
    from sdpa_b200 import instances
    from sdpa_b200.sdpa import SDPA
    meta = json.load(open(os.path.join(GOLDEN, "arrow.json")))["arrow"]
    xref = np.load(os.path.join(GOLDEN, "arrow.npz"))["arrow.xvec"]
    inst = instances.block_arrow_sdp()
    res = {}
    for mode in ("auto", "dense"):
        if mode == "dense":
            monkeypatch.setenv("SDPAB_SCHUR", "dense")
        else:
            monkeypatch.delenv("SDPAB_SCHUR", raising=False)
        s = SDPA()
        s.inputProblem(inst)
        s.solve()
        res[mode] = (s.getPhaseString(), s.getIteration(), s.getPrimalObj(), s.getDualObj(),
                     s.getResultXVec().copy(), s.schurPattern())
    phase, iters, pobj, dobj, x, (sparse, pairs, dense_pairs) = res["auto"]
    assert sparse and pairs < 0.6 * dense_pairs, (pairs, dense_pairs)
    assert phase == "pdOPT"
    assert abs(iters - meta["iterations"]) <= 1
    assert rel(pobj, meta["primal_obj"]) < OBJ_TOL
    assert rel(dobj, meta["dual_obj"]) < OBJ_TOL
    assert np.max(np.abs(x - xref)) < X_TOL
    phase2, iters2, pobj2, dobj2, x2, (sparse2, _, _) = res["dense"]
    assert not sparse2 and phase2 == "pdOPT" and iters2 == iters
    assert rel(pobj2, pobj) < 1e-9 and rel(dobj2, dobj) < 1e-9
    assert np.max(np.abs(x2 - x)) < 1e-7


def test_constraint_order_on_a_shuffled_block_arrow(monkeypatch):
    """A block-arrow problem with its constraints in a shuffled order: in
    file order its symbolic Schur pattern is dense; the solver reorders the
    constraints (minimum degree / arrowhead), takes the tile-sparse
    factorisation, and returns x in the caller's order.  The result equals
    the solve in the caller's order with the dense factorisation
    (SDPAB_ORDER=natural, SDPAB_SCHUR=dense) to rounding."""
    from sdpa_b200 import instances
    from sdpa_b200.sdpa import SDPA
    inst = instances.block_arrow_sdp(shuffled=True)
    res = {}
    for mode in ("ordered", "natural"):
        if mode == "natural":
            monkeypatch.setenv("SDPAB_ORDER", "natural")
            monkeypatch.setenv("SDPAB_SCHUR", "dense")
        else:
            monkeypatch.delenv("SDPAB_ORDER", raising=False)
            monkeypatch.delenv("SDPAB_SCHUR", raising=False)
        s = SDPA()
        s.inputProblem(inst)
        s.solve()
        res[mode] = (s.getPhaseString(), s.getIteration(), s.getPrimalObj(), s.getDualObj(),
                     s.getResultXVec().copy(), s.schurPattern())
    ph, it, po, do, x, (sparse, pairs, dense_pairs) = res["ordered"]
    ph2, it2, po2, do2, x2, (sparse2, _, _) = res["natural"]
    assert ph == ph2 == "pdOPT" and sparse and not sparse2 and pairs < 0.6 * dense_pairs
    assert abs(it - it2) <= 1
    assert rel(po, po2) < 1e-8 and rel(do, do2) < 1e-8
    assert np.max(np.abs(x - x2)) < 1e-6
