"""The sdpa command-line driver (sdpa_b200/_lib/sdpa), the drop-in for the
reference executable (sdpa_exe.cpp): argument handling and error exits on
CPU; solves compared with the reference executable's own result files
(tests/golden/cli, made by tests/golden/make_golden.py) on the GPU."""
import json
import os
import shutil
import subprocess

import numpy as np
import pytest

from golden_util import GOLDEN, parse_result

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "sdpa_b200", "_lib", "sdpa")
CLI_DIR = os.path.join(GOLDEN, "cli")


def _run(args, cwd):
    return subprocess.run([CLI] + args, cwd=cwd, capture_output=True, text=True, timeout=300)


@pytest.fixture
def workdir(tmp_path):
    if not os.path.exists(CLI):
        pytest.fail("sdpa_b200/_lib/sdpa is not built (python -m sdpa_b200.build)")
    for f in os.listdir(CLI_DIR):
        shutil.copy(os.path.join(CLI_DIR, f), tmp_path / f)
    return tmp_path


def test_usage_without_arguments(workdir):
    r = _run([], workdir)
    assert r.returncode == 1
    assert "Please assign data file and output file" in r.stdout


def test_missing_data_file_is_an_error(workdir):
    r = _run(["-ds", "nothere.dat-s", "-o", "x.result", "-pt", "0"], workdir)
    assert r.returncode == 1
    assert "cannot read the data file" in r.stderr


def test_positional_style_reads_param_sdpa(workdir):
    # style 1 reads ./param.sdpa unless -pt is given, as the reference does
    os.remove(workdir / "param.sdpa")
    r = _run(["ex1.dat-s", "x.result"], workdir)
    assert r.returncode == 1
    assert "parameter file" in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("case", range(3))
def test_result_file_matches_reference_executable(workdir, case):
    runs = json.load(open(os.path.join(CLI_DIR, "runs.json")))
    args, result = runs[case]["args"], runs[case]["result"]
    ref = parse_result(open(os.path.join(CLI_DIR, result)).read())
    os.remove(workdir / result)
    r = _run(args, workdir)
    assert r.returncode == 0, r.stderr
    ours = parse_result(open(workdir / result).read())
    # same layout line for line (numbers masked; dates dropped)
    assert ours["layout"] == ref["layout"]
    assert ours["info"]["phase.value"] == ref["info"]["phase.value"]
    assert ours["info"]["Iteration"] == ref["info"]["Iteration"]
    for k in ("objValPrimal", "objValDual"):
        a, b = float(ours["info"][k]), float(ref["info"][k])
        assert abs(a - b) <= 1e-6 * max(1.0, abs(b)), k
    # the iteration table: mu, objectives and beta along the same path
    assert len(ours["table"]) == len(ref["table"])
    for ro, rr in zip(ours["table"], ref["table"]):
        for c in (1, 4, 5, 8):
            assert abs(ro[c] - rr[c]) <= 0.02 * abs(rr[c]) + 1e-8, (ro, rr)
    # printed solutions (%+8.3e: four significant digits)
    for key in ("xVec", "xMat", "yMat"):
        a, b = np.array(ours[key]), np.array(ref[key])
        assert a.shape == b.shape, key
        assert np.all(np.abs(a - b) <= 2e-3 * np.abs(b) + 1e-5), key
    if ref["dimacs"]:
        # IO::computeDimacs values, computed on the GPU here
        assert set(ours["dimacs"]) == set(ref["dimacs"])
        od, rd = ours["dimacs"], ref["dimacs"]
        # err1, err3: residual norms at the rounding level on both sides
        for k in ("err1", "err3"):
            assert od[k] <= 1e-12 and rd[k] <= 1e-12, (k, od[k], rd[k])
        # err2, err4: zero while X and Z are positive definite
        for k in ("err2", "err4"):
            assert abs(od[k] - rd[k]) <= 1e-12, (k, od[k], rd[k])
        # err5, err6: relative gap and X.Z (= nDim mu) at the final iterate,
        # within the iteration table's own mu tolerance
        for k in ("err5", "err6"):
            assert abs(od[k] - rd[k]) <= 0.02 * abs(rd[k]) + 1e-13, (k, od[k], rd[k])
