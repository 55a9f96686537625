"""The reference's own library examples (libexample/example1-6.cpp of the
reference tree), compiled unchanged against include/sdpa_call.h and linked
with libsdpa_b200.so (oracle/Makefile `examples`), against the same
programs linked with the reference library: the same printed layout line
for line (numbers masked, the version banner excepted), the same phases and
iteration counts, objectives within 1e-6 and printed solutions within the
printed precision.  The ILP64 tree's copies of the same programs, compiled
with SDPA_INT = int64_t against libsdpa_b200_ilp64.so, must print the same."""
import os
import re
import shutil
import subprocess

import numpy as np
import pytest

from golden_util import GOLDEN, normalize_result_line, parse_result

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EX = os.path.join(ROOT, "oracle", "_ref", "examples")
ARGS = {1: [], 2: [], 3: [], 4: [], 5: ["ex1.dat-s", "out.result", "param.sdpa"],
        6: ["ex1.dat-s", "ex1.ini-s", "param.sdpa"]}
NUM = re.compile(r"[+-]?(?:\d+\.?\d*|\.\d+)(?:[eE][+-]?\d+)?")


def _run(binary, args, cwd):
    r = subprocess.run([binary] + args, cwd=cwd, capture_output=True, text=True, timeout=300,
                       env=dict(os.environ, OMP_NUM_THREADS="1", OPENBLAS_NUM_THREADS="1"))
    assert r.returncode == 0, (binary, r.stderr[-2000:])
    return r.stdout


def _values(text, key):
    return [float(NUM.findall(ln.split("=", 1)[1])[0]) for ln in text.splitlines()
            if ln.split("=")[0].strip() == key and "=" in ln]


@pytest.mark.parametrize("variant", ["b200", "b200_ilp64"])
@pytest.mark.parametrize("e", sorted(ARGS))
def test_reference_example_runs_unchanged_on_b200(e, variant, tmp_path):
    ref_bin = os.path.join(EX, f"ref_example{e}")
    ours_bin = os.path.join(EX, f"{variant}_example{e}")
    if not (os.path.exists(ref_bin) and os.path.exists(ours_bin)):
        pytest.skip("reference examples not built (make -C oracle examples needs the reference sources)")
    dirs = {}
    for who in ("ref", "ours"):
        d = tmp_path / who
        d.mkdir()
        for f in os.listdir(os.path.join(GOLDEN, "cli")):
            shutil.copy(os.path.join(GOLDEN, "cli", f), d / f)
        dirs[who] = d
    ref = _run(ref_bin, ARGS[e], dirs["ref"])
    ours = _run(ours_bin, ARGS[e], dirs["ours"])
    drop = lambda t: [normalize_result_line(ln) for ln in t.splitlines() if "has been developed" not in ln
                      and "sdpa_b200" not in ln]
    assert drop(ours) == drop(ref)
    for key in ("phase.value", "Phase"):
        assert [ln for ln in ours.splitlines() if ln.startswith(key)] == \
               [ln for ln in ref.splitlines() if ln.startswith(key)]
    assert _values(ours, "Iteration") == _values(ref, "Iteration")
    for key in ("objValPrimal", "objValDual"):
        a, b = np.array(_values(ours, key)), np.array(_values(ref, key))
        assert a.shape == b.shape
        assert np.all(np.abs(a - b) <= 1e-6 * np.maximum(1.0, np.abs(b))), key
    # every number printed after the first "xVec" (solutions at %+8.3e)
    tail = lambda t: np.array([float(x) for x in NUM.findall(t[t.index("xVec"):])]) if "xVec" in t else np.zeros(0)
    a, b = tail(ours), tail(ref)
    assert a.shape == b.shape
    assert np.all(np.abs(a - b) <= 2e-3 * np.abs(b) + 1e-5)
    # a result file written by the example (example 5): the same comparison
    if "out.result" in ARGS[e]:
        ro = parse_result(open(dirs["ours"] / "out.result").read())
        rr = parse_result(open(dirs["ref"] / "out.result").read())
        assert ro["layout"] == rr["layout"]
        assert ro["info"]["phase.value"] == rr["info"]["phase.value"]
        for k in ("objValPrimal", "objValDual"):
            x, y = float(ro["info"][k]), float(rr["info"][k])
            assert abs(x - y) <= 1e-6 * max(1.0, abs(y)), k
        for k in ("xVec", "xMat", "yMat"):
            x, y = np.array(ro[k]), np.array(rr[k])
            assert x.shape == y.shape and np.all(np.abs(x - y) <= 2e-3 * np.abs(y) + 1e-5), k
