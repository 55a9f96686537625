"""Runs the REFERENCE solver on a batch of instances (test infrastructure and
CPU baseline only; never imported by the product).

`oracle/_ref/ref_batch` is the reference SDPA 7.4.4 (LP64 tree) compiled from
its own sources by oracle/Makefile and driven through its own class SDPA
(sdpa_call.h:91-267), the sequence of the reference CLI (sdpa_exe.cpp:224-343).
This module writes the instances as .dat-s files, runs ref_batch with one
single-threaded process per core, and parses one RESULT and one XVEC line per
instance (objectives, iterations, phase, SDPA's xVec from getResultXVec,
sdpa_call.cpp:668-672).

It also holds the parity bar used for paths that leave the reference's
iterate sequence (warm start, mixed precision): `x_within_reference_accuracy`.
"""
from __future__ import annotations

import os
import subprocess
import tempfile
import time
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_BATCH = os.path.join(HERE, "_ref", "ref_batch")

# param.sdpa with the reference's default values (Parameter::setDefaultParameter,
# sdpa_parts.cpp:182-224: epsilonStar = epsilonDash = 1e-7)
PARAM_DEFAULT = """100 maxIteration
1.0E-7 epsilonStar
1.0E2 lambdaStar
2.0 omegaStar
-1.0E5 lowerBound
1.0E5 upperBound
0.1 betaStar
0.2 betaBar
0.9 gammaStar
1.0E-7 epsilonDash
%+8.3e xPrint
%+8.3e XPrint
%+8.3e YPrint
%+10.16e infPrint
"""

# The same with epsilonStar 1e-11 / epsilonDash 1e-9: the reference's solution
# polished far past the default stopping test (x* of the parity bar below).
PARAM_TIGHT = (PARAM_DEFAULT.replace("100 maxIteration", "200 maxIteration")
               .replace("1.0E-7 epsilonStar", "1.0E-11 epsilonStar")
               .replace("1.0E-7 epsilonDash", "1.0E-9 epsilonDash"))

PHASES = {"noINFO": 0, "pFEAS": 1, "dFEAS": 2, "pdFEAS": 3, "pdINF": 4, "pFEAS_dINF": 5,
          "pINF_dFEAS": 6, "pdOPT": 7, "pUNBD": 8, "dUNBD": 9}


@dataclass
class RefRun:
    wall_s: float              # longest worker's summed initializeSolve + solve time
    process_wall_s: float      # the whole ref_batch run, parsing and start-up included
    iterations: np.ndarray
    phase: np.ndarray          # SDPA::getPhaseValue() codes (pdOPT = 7)
    primal_obj: np.ndarray
    dual_obj: np.ndarray
    x: list                    # xVec per instance


def available() -> bool:
    return os.path.exists(REF_BATCH)


def write_instances(instances, tmp: str) -> str:
    """Writes every instance as tmp/i<q>.dat-s and returns the list file."""
    paths = []
    for q, it in enumerate(instances):
        p = os.path.join(tmp, f"i{q}.dat-s")
        it.write(p)
        paths.append(p)
    lst = os.path.join(tmp, "list.txt")
    with open(lst, "w") as f:
        f.write("\n".join(paths))
    return lst


def run(instances=None, procs: int | None = None, param: str | None = None, tmp: str | None = None,
        count: int | None = None) -> RefRun:
    """Solves `instances` (or the `count` files already written to `tmp` by
    write_instances) with the reference, `procs` single-threaded processes.
    `param` is param.sdpa text (None: the reference's defaults)."""
    if not available():
        raise FileNotFoundError("oracle/_ref/ref_batch is not built (make -C oracle)")
    procs = procs or os.cpu_count() or 1
    own = tmp is None
    tdir = tempfile.mkdtemp() if own else tmp
    try:
        if instances is not None:
            lst = write_instances(instances, tdir)
            count = len(instances)
        else:
            lst = os.path.join(tdir, "list.txt")
        cmd = [REF_BATCH, "--procs", str(procs), "--xvec", "--list", lst]
        if param is not None:
            pp = os.path.join(tdir, "param.sdpa")
            with open(pp, "w") as f:
                f.write(param)
            cmd[1:1] = ["--param", pp]
        env = dict(os.environ, OMP_NUM_THREADS="1", OPENBLAS_NUM_THREADS="1")
        t0 = time.time()
        out = subprocess.run(cmd, capture_output=True, text=True, env=env, check=True).stdout
        pwall = time.time() - t0
    finally:
        if own:
            import shutil
            shutil.rmtree(tdir, ignore_errors=True)
    it = np.zeros(count, np.int32)
    ph = np.full(count, -1, np.int32)
    po = np.full(count, np.nan)
    do = np.full(count, np.nan)
    xs = [None] * count
    wall = None
    index = lambda f: int(os.path.basename(f)[1:].split(".")[0])
    for line in out.splitlines():
        t = line.split()
        if not t:
            continue
        if t[0] == "RESULT":
            q = index(t[1])
            it[q], ph[q] = int(t[2]), PHASES.get(t[3], -1)
            po[q], do[q] = float(t[4]), float(t[5])
        elif t[0] == "XVEC":
            q, m = index(t[1]), int(t[2])
            if len(t) != 3 + m:
                raise RuntimeError(f"ref_batch: malformed XVEC line for instance {q}")
            xs[q] = np.array([float(v) for v in t[3:]])
        elif t[0] == "WALL":
            wall = float(t[1])
    missing = [q for q in range(count) if xs[q] is None or ph[q] < 0]
    if missing or wall is None:
        raise RuntimeError(f"ref_batch: no result for {len(missing)} instances")
    return RefRun(wall, pwall, it, ph, po, do, xs)


def x_within_reference_accuracy(x, x_ref, x_tight, tol=1e-5) -> bool:
    """Parity bar on x for paths that leave the reference's iterate sequence
    (warm start, mixed precision).  At the default stopping test the
    reference's own x is determined only to |x_ref - x*| (x* its solution at
    epsilonStar 1e-11; up to 1.5e-4 on batched MaxCut, more where the optimal
    face is not a point), so such a path must land at least as close to x*
    as the reference does, up to `tol`."""
    return float(np.max(np.abs(x - x_tight))) <= float(np.max(np.abs(x_ref - x_tight))) + tol


def parity_counts(primal, dual, xs, ref: RefRun, tight: RefRun | None = None, phase=None) -> dict:
    """Per-instance comparison with the reference's results on the same
    inputs: objectives within 1e-6 relative (both), x within 1e-5 (max abs),
    and, for the instances outside 1e-5, whether x passes the reference-
    accuracy bar against the tight solution.  With `phase` (the solver's
    phase codes) also the phase agreement, and the objective and x counts
    over the instances that both solvers end at pdOPT: an instance that the
    reference stops short of optimal (pdFEAS after a step too short to
    continue) ends where rounding decides, for the reference's own build as
    for any other, and its x is not determined."""
    n = len(xs)
    rel = lambda a, b: np.abs(a - b) / np.maximum(1.0, np.abs(b))
    rp = rel(np.asarray(primal), ref.primal_obj)
    rd = rel(np.asarray(dual), ref.dual_obj)
    dx = np.array([float(np.max(np.abs(np.asarray(xs[q]) - ref.x[q]))) for q in range(n)])
    obj_ok = (rp <= 1e-6) & (rd <= 1e-6)
    x_ok = dx <= 1e-5
    out = {"count": n, "objectives_within_1e-6": int(obj_ok.sum()),
           "max_rel_objective_diff": float(max(rp.max(), rd.max())),
           "x_within_1e-5": int(x_ok.sum()), "max_abs_x_diff": float(dx.max()),
           "reference_pdOPT": int(np.sum(ref.phase == 7))}
    if tight is not None:
        acc = np.array([x_ok[q] or x_within_reference_accuracy(np.asarray(xs[q]), ref.x[q], tight.x[q])
                        for q in range(n)])
        out["x_only_within_reference_accuracy"] = int(np.sum(acc & ~x_ok))
        out["x_failing_both_bars"] = int(np.sum(~acc))
    if phase is not None:
        ph = np.asarray(phase)
        both = (ph == 7) & (ref.phase == 7)
        out["phase_equal"] = int(np.sum(ph == ref.phase))
        out["both_pdOPT"] = int(both.sum())
        out["objectives_within_1e-6_both_pdOPT"] = int(np.sum(obj_ok & both))
        out["x_within_1e-5_both_pdOPT"] = int(np.sum(x_ok & both))
        if both.any():
            out["max_abs_x_diff_both_pdOPT"] = float(dx[both].max())
        if tight is not None:
            out["x_failing_both_bars_both_pdOPT"] = int(np.sum(~acc & both))
    return out
