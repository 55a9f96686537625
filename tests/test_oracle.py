"""The CPU oracle (oracle/sdpa_oracle.py) pinned against the reference
solver's own results (tests/golden, produced by oracle/_ref from the reference
sources) and the known answers printed in the reference manual."""
import importlib.util
import os

import numpy as np
import pytest

from golden_util import GOLDEN, known_answers, rel, small
from oracle import sdpa_oracle as O

_spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLDEN, "make_golden.py"))
MG = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(MG)


def test_manual_known_answers():
    ka = known_answers()
    for name, inst in (("example1", MG.example1()), ("example2", MG.example2())):
        r = O.solve(O.parse_dats(inst.to_dats()))
        man = ka["manual"][name]
        assert r.iterations == man["iterations"]
        assert O.PHASE_NAMES[r.phase] == "pdOPT"
        assert rel(r.primal_obj, man["primal_obj"]) < 1e-9
        assert rel(r.dual_obj, man["dual_obj"]) < 1e-9
        ref = ka["reference_default"][name]
        assert rel(r.primal_obj, ref["primal_obj"]) < 1e-12
        assert np.allclose(r.xvec, ref["xvec"], atol=1e-9, rtol=0)


def test_param_file_epsilon_1e8():
    ka = known_answers()
    p = O.Params(maxIteration=200, epsilonStar=1e-8, lambdaStar=1e2, omegaStar=2.0, lowerBound=-1e20,
                 upperBound=1e20, betaStar=0.1, betaBar=0.2, gammaStar=0.9, epsilonDash=1e-8)
    for name, inst in (("example1", MG.example1()), ("example2", MG.example2())):
        r = O.solve(O.parse_dats(inst.to_dats()), p)
        ref = ka["reference_param_1e-8"][name]
        assert r.iterations == ref["iterations"]
        assert rel(r.primal_obj, ref["primal_obj"]) < 1e-10


@pytest.mark.parametrize("name", ["mc20", "mc50w", "lt20", "lt40", "rnd40", "ex2", "bmc0", "bmc1",
                                  "bmc5"])
def test_oracle_matches_reference(name):
    meta, arr = small()
    inst = dict(MG.small_cases())[name]
    r = O.solve(O.parse_dats(inst.to_dats()))
    g = meta[name]
    assert O.PHASE_NAMES[r.phase] == g["phase"]
    assert r.iterations == g["iterations"]
    assert rel(r.primal_obj, g["primal_obj"]) < 1e-9
    assert rel(r.dual_obj, g["dual_obj"]) < 1e-9
    assert np.max(np.abs(r.xvec - arr[name + ".xvec"])) < 1e-6


def test_dats_roundtrip():
    inst = MG.example2()
    P = O.parse_dats(inst.to_dats())
    assert P.m == 5 and P.blocks == [2, 3, -2]
    assert len(P.entries[0]) == len([1 for k in inst.k if k == 0])


def test_headline_fixture_matches_oracle_and_runner():
    """The headline fixture (reference results for the benchmark's seeds
    0..511) agrees with the numpy restatement on a few seeds, and, where the
    reference build is present, with a fresh reference run through
    oracle.ref_runner (the path bench.py's reference arm takes)."""
    import json
    from oracle import ref_runner as R
    from sdpa_b200 import instances as I
    meta = json.load(open(os.path.join(GOLDEN, "headline.json")))
    arr = np.load(os.path.join(GOLDEN, "headline.npz"))
    seeds = [0, 1, 7, 300]
    its = [I.batch_maxcut(s, 20, 120) for s in seeds]
    for s, it in zip(seeds, its[:2]):
        r = O.solve(O.parse_dats(it.to_dats()))
        assert r.iterations == meta["iterations"][s]
        assert rel(r.primal_obj, meta["primal_obj"][s]) < 1e-10
        assert np.max(np.abs(r.xvec - arr[f"bmc{s}.xvec"])) < 1e-7
    if not R.available():
        pytest.skip("oracle/_ref/ref_batch not built")
    run = R.run(its, procs=2)
    for q, s in enumerate(seeds):
        assert run.phase[q] == 7 and run.iterations[q] == meta["iterations"][s]
        assert run.primal_obj[q] == meta["primal_obj"][s] and run.dual_obj[q] == meta["dual_obj"][s]
        assert np.array_equal(run.x[q], arr[f"bmc{s}.xvec"])
    pc = R.parity_counts(run.primal_obj, run.dual_obj, run.x, run, run)
    assert pc["objectives_within_1e-6"] == len(seeds) and pc["x_failing_both_bars"] == 0


def test_parity_counts_split_by_phase():
    """Instances the reference stops short of pdOPT are counted apart: their
    x is not determined, so a large x difference there is reported but does
    not enter the both-pdOPT counts."""
    from oracle import ref_runner as R
    ref = R.RefRun(wall_s=1.0, process_wall_s=1.0, iterations=np.array([9, 9, 9]),
                   phase=np.array([7, 7, 3]), primal_obj=np.array([1.0, 2.0, 3.0]),
                   dual_obj=np.array([1.0, 2.0, 3.0]),
                   x=[np.array([0.5, 0.25]), np.array([1.0, 2.0]), np.array([1.0, 1.0])])
    ours_x = [np.array([0.5, 0.25 + 4e-6]), np.array([1.0, 2.0 + 3e-5]), np.array([1.0, 900.0])]
    pc = R.parity_counts([1.0, 2.0, 3.0 + 1e-3], [1.0, 2.0, 3.0], ours_x, ref, phase=[7, 7, 7])
    assert pc["objectives_within_1e-6"] == 2 and pc["x_within_1e-5"] == 1
    assert pc["phase_equal"] == 2 and pc["both_pdOPT"] == 2
    assert pc["objectives_within_1e-6_both_pdOPT"] == 2 and pc["x_within_1e-5_both_pdOPT"] == 1
    assert pc["max_abs_x_diff"] == pytest.approx(899.0)
    assert pc["max_abs_x_diff_both_pdOPT"] == pytest.approx(3e-5)
