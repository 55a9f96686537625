"""Regenerates the golden fixtures in this directory by running the REFERENCE
solver (oracle/_ref/ref_batch, compiled from the reference sources by
oracle/Makefile) on seeded instances from sdpa_b200.instances.

Run here (where the reference sources exist):
    make -C oracle && python tests/golden/make_golden.py [--large]

Fixtures (all from the reference's own output, never hand-written):
  known_answers.json   example1/example2 of the reference manual, with the
                       manual's printed values and the reference's run here
  small.npz / small.json   small instances: objectives, iterations, phase, x,
                       and the final Y/X blocks (MaxCut, Lovasz theta, random
                       SDP with an LP block, batched-MaxCut seeds 0..63)
  mc100_trace.json     per-iteration (mu, objP, objD, alphaP, alphaD, beta)
                       of MaxCut G(100, 0.1) seed 1 at epsilonStar = 1e-7
  blocks.json / blocks.npz  (also alone with --blocks) batched multi-block
                       instances blk0..blk31 and the dense-constraint
                       single-block instances dns0..dns7: objectives,
                       iterations, phase, x; X and Y for blk0..blk7, dns*
  arrow.json / arrow.npz  (also alone with --arrow) a many-block SDP with a
                       sparse Schur matrix, from the numpy restatement
                       (the reference's sparse path needs MUMPS)
  large.json / large.npz  (--large) Lovasz theta G(200, 0.5) seed 1 and the
                       random m=2000 SDP seed 1: objectives, iterations, x
  headline.json / headline.npz  (also alone with --headline) the first 512
                       instances of the 4096-instance batched MaxCut benchmark
                       (seeds 0..511, n ~ U{20..120}): objectives, iterations,
                       phase and x at the default parameters, and x at
                       epsilonStar 1e-11 (x* of the reference-accuracy bar)
  tcfb.json / tcfb.npz  (also alone with --tcfb) a random SDP with m = 300 and
                       an order-80 block (the mixed mode's tensor-core paths):
                       objectives, x, and x at epsilonStar 1e-11
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from sdpa_b200 import instances as inst  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref", "ref_batch")
REF_CLI = os.path.join(ROOT, "oracle", "_ref", "sdpa")  # the reference's own executable (sdpa_exe.cpp)


def example1():
    """Example 1 of the reference manual: m=3, one 2x2 block."""
    E = [(0, 1, 1, 1, -11.0), (0, 1, 2, 2, 23.0), (1, 1, 1, 1, 10.0), (1, 1, 1, 2, 4.0),
         (2, 1, 2, 2, -8.0), (3, 1, 1, 2, -8.0), (3, 1, 2, 2, -2.0)]
    a = np.array(E, dtype=object)
    return inst.Instance(m=3, blocks=[2], c=np.array([48.0, -8.0, 20.0]),
                         k=a[:, 0].astype(np.int32), l=a[:, 1].astype(np.int32),
                         i=a[:, 2].astype(np.int32), j=a[:, 3].astype(np.int32),
                         v=a[:, 4].astype(float), name="example1")


def example2():
    """Example 2 of the reference manual: m=5, blocks {2, 3, -2}."""
    F = [
        ([[-1.4, -3.2], [-3.2, -28]], [[15, -12, 2.1], [-12, 16, -3.8], [2.1, -3.8, 15]], [1.8, -4.0]),
        ([[0.5, 5.2], [5.2, -5.3]], [[7.8, -2.4, 6.0], [-2.4, 4.2, 6.5], [6.0, 6.5, 2.1]], [-4.5, -3.5]),
        ([[1.7, 7.0], [7.0, -9.3]], [[-1.9, -0.9, -1.3], [-0.9, -0.8, -2.1], [-1.3, -2.1, 4.0]], [-0.2, -3.7]),
        ([[6.3, -7.5], [-7.5, -3.3]], [[0.2, 8.8, 5.4], [8.8, 3.4, -0.4], [5.4, -0.4, 7.5]], [-3.3, -4.0]),
        ([[-2.4, -2.5], [-2.5, -2.9]], [[3.4, -3.2, -4.5], [-3.2, 3.0, -4.8], [-4.5, -4.8, 3.6]], [4.8, 9.7]),
        ([[-6.5, -5.4], [-5.4, -6.6]], [[6.7, -7.2, -3.6], [-7.2, 7.3, -3.0], [-3.6, -3.0, -1.4]], [6.1, -1.5]),
    ]
    E = []
    for k, (b1, b2, lp) in enumerate(F):
        for l, B in ((1, b1), (2, b2)):
            B = np.array(B, dtype=float)
            for r in range(B.shape[0]):
                for s in range(r, B.shape[0]):
                    if B[r, s] != 0.0:
                        E.append((k, l, r + 1, s + 1, B[r, s]))
        for t, v in enumerate(lp):
            if v != 0.0:
                E.append((k, 3, t + 1, t + 1, float(v)))
    a = np.array(E, dtype=object)
    return inst.Instance(m=5, blocks=[2, 3, -2], c=np.array([1.1, -10, 6.6, 19, 4.1]),
                         k=a[:, 0].astype(np.int32), l=a[:, 1].astype(np.int32),
                         i=a[:, 2].astype(np.int32), j=a[:, 3].astype(np.int32),
                         v=a[:, 4].astype(float), name="example2")


PARAM_1E8 = """200 maxIteration
1.0E-8 epsilonStar
1.0E2 lambdaStar
2.0 omegaStar
-1.0E20 lowerBound
1.0E20 upperBound
0.1 betaStar
0.2 betaBar
0.9 gammaStar
1.0E-8 epsilonDash
%+10.16e xPrint
%+10.16e XPrint
%+10.16e YPrint
%+10.16e infPrint
"""


# epsilonStar 1e-11: the reference's own solution polished far past the
# default stopping test, the optimum that paths which leave the reference's
# iterate sequence (warm start, mixed precision) are compared against.
PARAM_TIGHT = PARAM_1E8.replace("1.0E-8 epsilonStar", "1.0E-11 epsilonStar").replace(
    "1.0E-8 epsilonDash", "1.0E-9 epsilonDash")


def heldout_cases(count=64):
    """MaxCut SDPs of the warm-start held-out seeds (300000.., n ~ U{50..200})."""
    return [(f"ws{s}", inst.batch_maxcut(s, 50, 200)) for s in range(300000, 300000 + count)]


def run_ref(instances, tmp, param=None, trace=False, procs=1, threads=1):
    paths = []
    for q, it in enumerate(instances):
        p = os.path.join(tmp, f"i{q}.dat-s")
        it.write(p)
        paths.append(p)
    cmd = [REF, "--dump", tmp] + (["--param", param] if param else []) + (["--trace"] if trace else [])
    cmd += ["--procs", str(procs)] + paths
    env = dict(os.environ, OMP_NUM_THREADS=str(threads), OPENBLAS_NUM_THREADS=str(threads))
    out = subprocess.run(cmd, capture_output=True, text=True, env=env, check=True).stdout
    res, tr = {}, {}
    for line in out.splitlines():
        t = line.split()
        if t[0] == "RESULT":
            res[t[1]] = dict(iterations=int(t[2]), phase=t[3], primal_obj=float(t[4]),
                             dual_obj=float(t[5]), seconds=float(t[6]))
        elif t[0] == "TRACE" and len(t) >= 11 and t[2].isdigit():
            tr.setdefault(t[1], []).append([float(x) for x in t[3:11]])
    outl = []
    for q, it in enumerate(instances):
        p = paths[q]
        r = res[p]
        b = os.path.join(tmp, f"i{q}")
        r["xvec"] = np.fromfile(b + ".xvec.bin")
        r["X"], r["Y"] = [], []
        for l, s in enumerate(it.blocks, start=1):
            n = s * s if s > 1 else abs(s)
            r["X"].append(np.fromfile(b + f".X{l}.bin"))
            r["Y"].append(np.fromfile(b + f".Y{l}.bin"))
        if trace:
            r["trace"] = tr.get(p, [])
        outl.append(r)
    return outl


def write_dense(it, path):
    """The instance in SDPA's dense .dat format (IO::read dense branch,
    sdpa_io.cpp:540-604): header, then F0..Fm, each block as a full matrix
    (SDP) or its diagonal (LP)."""
    mats = []
    for k in range(it.m + 1):
        blocks = []
        for l, bs in enumerate(it.blocks, start=1):
            n = abs(int(bs))
            blocks.append(np.zeros((n, n)) if bs > 0 else np.zeros(n))
        for q in range(it.k.size):
            if int(it.k[q]) != k:
                continue
            B = blocks[int(it.l[q]) - 1]
            r, c = int(it.i[q]) - 1, int(it.j[q]) - 1
            if B.ndim == 2:
                B[r, c] = B[c, r] = float(it.v[q])
            else:
                B[r] = float(it.v[q])
        mats.append(blocks)
    fmt = lambda a: ",".join(repr(float(x)) for x in a)
    out = [f'"{it.name} (dense)"', f"{it.m} = mDIM", f"{len(it.blocks)} = nBLOCK",
           " ".join(str(int(b)) for b in it.blocks) + " = bLOCKsTRUCT", "{" + fmt(it.c) + "}"]
    for blocks in mats:
        parts = []
        for B in blocks:
            if B.ndim == 2:
                parts.append("{ " + ", ".join("{" + fmt(row) + "}" for row in B) + " }")
            else:
                parts.append("{" + fmt(B) + "}")
        out.append("{ " + " ".join(parts) + " }")
    with open(path, "w") as f:
        f.write("\n".join(out) + "\n")


def cli_fixtures():
    """Inputs and the reference executable's result files for the command-line
    driver test (tests/golden/cli): example 1 sparse with -pt 0, example 2
    dense in the positional style with -pt 0 and -dimacs, example 1 with a
    parameter file (epsilonStar 1e-8)."""
    d = os.path.join(HERE, "cli")
    os.makedirs(d, exist_ok=True)
    example1().write(os.path.join(d, "ex1.dat-s"))
    write_dense(example2(), os.path.join(d, "ex2.dat"))
    with open(os.path.join(d, "param.sdpa"), "w") as f:
        f.write(PARAM_1E8)
    # an interior initial point for example 1 (x, then user X and Y entries)
    with open(os.path.join(d, "ex1.ini-s"), "w") as f:
        f.write("0.0 0.0 0.0\n1 1 1 1 10.0\n1 1 2 2 10.0\n2 1 1 1 10.0\n2 1 2 2 10.0\n")
    runs = [(["-ds", "ex1.dat-s", "-o", "ex1.result", "-pt", "0"], "ex1.result"),
            (["ex2.dat", "ex2.result", "-pt", "0", "-dimacs"], "ex2.result"),
            (["-ds", "ex1.dat-s", "-o", "ex1p.result", "-p", "param.sdpa"], "ex1p.result")]
    env = dict(os.environ, OMP_NUM_THREADS="1", OPENBLAS_NUM_THREADS="1")
    for args, _ in runs:
        subprocess.run([REF_CLI] + args, cwd=d, env=env, check=True, capture_output=True)
    with open(os.path.join(d, "runs.json"), "w") as f:
        json.dump([{"args": a, "result": r} for a, r in runs], f, indent=1)


def small_cases():
    cases = [("mc100", inst.maxcut(100, 0.1, 1)), ("mc20", inst.maxcut(20, 0.3, 1)),
             ("mc50w", inst.maxcut(50, 0.2, 5, unit_weights=False)),
             ("lt20", inst.lovasz_theta(20, 0.5, 1)), ("lt40", inst.lovasz_theta(40, 0.3, 2)),
             ("rnd40", inst.random_sdp(m=40, n=12, nlp=5, density=0.1, seed=3)),
             ("rnd120", inst.random_sdp(m=120, n=30, nlp=8, density=0.05, seed=4)),
             ("ex2", example2())]
    cases += [(f"bmc{s}", inst.batch_maxcut(s)) for s in range(64)]
    return cases


def block_cases(count=32):
    """Batched multi-block instances (several SDP blocks and an LP block)."""
    return [(f"blk{s}", inst.batch_block_sdp(s)) for s in range(count)]


def dense_cases(count=8):
    """Single-block instances whose constraints have many entries (more than
    2n NonZeroEffect), which the batched solver assembles by F1."""
    out = []
    for s in range(count):
        n = 16 + 4 * s
        out.append((f"dns{s}", inst.random_block_sdp(m=12 + 2 * s, blocks=[n], density=0.5, seed=500 + s,
                                                      name=f"dense-constraint sdp n={n} seed {500 + s}")))
    return out


def block_fixtures(tmp):
    """blocks.json / blocks.npz: the reference's results (objectives,
    iterations, phase, x; every block of X and Y for blk0..blk7) on
    block_cases()."""
    cases = block_cases() + dense_cases()
    res = run_ref([c[1] for c in cases], tmp, procs=8)
    meta, arrays = {}, {}
    for (name, it), r in zip(cases, res):
        meta[name] = {k: r[k] for k in ("iterations", "phase", "primal_obj", "dual_obj")}
        arrays[name + ".xvec"] = r["xvec"]
        if name.startswith("dns") or int(name[3:]) < 8:
            for l in range(len(it.blocks)):
                arrays[name + f".X{l + 1}"] = r["X"][l]
                arrays[name + f".Y{l + 1}"] = r["Y"][l]
    with open(os.path.join(HERE, "blocks.json"), "w") as f:
        json.dump(meta, f, indent=1)
    np.savez_compressed(os.path.join(HERE, "blocks.npz"), **arrays)


def arrow_fixtures():
    """arrow.json / arrow.npz: a many-block SDP whose Schur matrix is sparse
    (block-diagonal with a dense border).  The reference takes its MUMPS
    sparse-Schur path on it, which is not built here (MUMPS is absent and
    stubbed), so these values come from the numpy restatement
    (oracle/sdpa_oracle.py) of the reference's algorithm."""
    from oracle import sdpa_oracle as O
    it = inst.block_arrow_sdp()
    r = O.solve(O.parse_dats(it.to_dats()))
    meta = {"arrow": {"iterations": r.iterations, "phase": O.PHASE_NAMES[r.phase], "primal_obj": r.primal_obj,
                      "dual_obj": r.dual_obj, "source": "numpy restatement (oracle/sdpa_oracle.py)"}}
    with open(os.path.join(HERE, "arrow.json"), "w") as f:
        json.dump(meta, f, indent=1)
    np.savez_compressed(os.path.join(HERE, "arrow.npz"), **{"arrow.xvec": r.xvec})


HEADLINE_SEEDS = 512


def headline_fixtures():
    """Reference results for the benchmark's batched MaxCut seeds 0..511:
    the headline configuration (learned warm start, mixed precision) is
    compared with these in tests/test_headline_parity_gpu.py."""
    from oracle import ref_runner as R
    its = [inst.batch_maxcut(s, 20, 120) for s in range(HEADLINE_SEEDS)]
    rd = R.run(its)
    rt = R.run(its, param=R.PARAM_TIGHT)
    meta = {"seeds": [0, HEADLINE_SEEDS], "generator": "sdpa_b200.instances.batch_maxcut(seed, 20, 120)",
            "iterations": rd.iterations.tolist(), "phase": rd.phase.tolist(),
            "primal_obj": rd.primal_obj.tolist(), "dual_obj": rd.dual_obj.tolist(),
            "tight_phase": rt.phase.tolist(), "tight_param": "epsilonStar 1e-11, epsilonDash 1e-9"}
    arrays = {}
    for s in range(HEADLINE_SEEDS):
        arrays[f"bmc{s}.xvec"] = rd.x[s]
        arrays[f"bmc{s}.tight"] = rt.x[s]
    with open(os.path.join(HERE, "headline.json"), "w") as f:
        json.dump(meta, f)
    np.savez_compressed(os.path.join(HERE, "headline.npz"), **arrays)


def tc_fallback_fixtures():
    """Reference results (default and epsilonStar 1e-11 x) of a random SDP
    large enough for the mixed mode's tensor-core paths (m >= 256, F1
    constraints in a block of order > 64): the fall-back test of those
    paths compares with these."""
    from oracle import ref_runner as R
    it = inst.random_sdp(m=300, n=80, nlp=6, density=0.1, seed=11)
    rd = R.run([it], procs=1)
    rt = R.run([it], procs=1, param=R.PARAM_TIGHT)
    meta = {"rnd300": {"iterations": int(rd.iterations[0]), "phase": int(rd.phase[0]),
                       "primal_obj": float(rd.primal_obj[0]), "dual_obj": float(rd.dual_obj[0]),
                       "generator": "sdpa_b200.instances.random_sdp(m=300, n=80, nlp=6, density=0.1, seed=11)"}}
    with open(os.path.join(HERE, "tcfb.json"), "w") as f:
        json.dump(meta, f, indent=1)
    np.savez_compressed(os.path.join(HERE, "tcfb.npz"), **{"rnd300.xvec": rd.x[0], "rnd300.tight": rt.x[0]})


def main():
    large = "--large" in sys.argv
    if "--tcfb" in sys.argv:
        tc_fallback_fixtures()
        return
    if "--headline" in sys.argv:
        headline_fixtures()
        return
    if "--arrow" in sys.argv:
        arrow_fixtures()
        return
    if "--blocks" in sys.argv:
        with tempfile.TemporaryDirectory() as tmp:
            block_fixtures(tmp)
        return
    with tempfile.TemporaryDirectory() as tmp:
        ppath = os.path.join(tmp, "param_1e-8.sdpa")
        with open(ppath, "w") as f:
            f.write(PARAM_1E8)
        # known answers (manual section 6) + reference runs here
        r_def = run_ref([example1(), example2()], tmp)
        r_p8 = run_ref([example1(), example2()], tmp, param=ppath)
        ka = {"manual": {"example1": {"iterations": 10, "primal_obj": -4.1899996163866390e+01,
                                      "dual_obj": -4.1899999999999999e+01, "epsilonStar": 1e-7},
                         "example2": {"iterations": 13, "primal_obj": 3.2062693405e+01,
                                      "dual_obj": 3.2062692354e+01, "epsilonStar": 1e-7}},
              "reference_default": {}, "reference_param_1e-8": {}}
        for name, a, b in zip(["example1", "example2"], r_def, r_p8):
            for key, r in (("reference_default", a), ("reference_param_1e-8", b)):
                ka[key][name] = {k: (v.tolist() if isinstance(v, np.ndarray) else v)
                                 for k, v in r.items() if k in ("iterations", "phase", "primal_obj",
                                                                "dual_obj", "xvec")}
        with open(os.path.join(HERE, "known_answers.json"), "w") as f:
            json.dump(ka, f, indent=1)

        cases = small_cases()
        res = run_ref([c[1] for c in cases], tmp, procs=8)
        meta, arrays = {}, {}
        for (name, it), r in zip(cases, res):
            meta[name] = {k: r[k] for k in ("iterations", "phase", "primal_obj", "dual_obj")}
            arrays[name + ".xvec"] = r["xvec"]
            if it.blocks[0] <= 50 or name == "mc100":
                for l in range(len(it.blocks)):
                    arrays[name + f".X{l + 1}"] = r["X"][l]
                    arrays[name + f".Y{l + 1}"] = r["Y"][l]
        with open(os.path.join(HERE, "small.json"), "w") as f:
            json.dump(meta, f, indent=1)
        np.savez_compressed(os.path.join(HERE, "small.npz"), **arrays)

        tr = run_ref([inst.maxcut(100, 0.1, 1)], tmp, trace=True)[0]
        with open(os.path.join(HERE, "mc100_trace.json"), "w") as f:
            json.dump({"columns": ["mu", "thetaP", "thetaD", "objP", "objD",
                                   "alphaP", "alphaD", "beta"], "rows": tr["trace"],
                       "iterations": tr["iterations"]}, f, indent=1)

        # tight solutions (and default ones for the held-out set)
        tpath = os.path.join(tmp, "param_tight.sdpa")
        with open(tpath, "w") as f:
            f.write(PARAM_TIGHT)
        tcases = cases + heldout_cases()
        rt = run_ref([c[1] for c in tcases], tmp, param=tpath, procs=8)
        ho = heldout_cases()
        rd = run_ref([c[1] for c in ho], tmp, procs=8)
        meta, arrays = {"heldout_default": {}, "tight": {}}, {}
        for (name, it), r in zip(tcases, rt):
            meta["tight"][name] = {k: r[k] for k in ("iterations", "phase", "primal_obj", "dual_obj")}
            arrays[name + ".tight"] = r["xvec"]
        for (name, it), r in zip(ho, rd):
            meta["heldout_default"][name] = {k: r[k] for k in ("iterations", "phase", "primal_obj", "dual_obj")}
            arrays[name + ".xvec"] = r["xvec"]
        with open(os.path.join(HERE, "tight.json"), "w") as f:
            json.dump(meta, f, indent=1)
        np.savez_compressed(os.path.join(HERE, "tight.npz"), **arrays)

        cli_fixtures()
        block_fixtures(tmp)
        arrow_fixtures()
        headline_fixtures()
        tc_fallback_fixtures()

        if large:
            big = [("lt200", inst.lovasz_theta(200, 0.5, 1)), ("rnd2000", inst.random_sdp(seed=1))]
            meta, arrays = {}, {}
            for name, it in big:
                r = run_ref([it], tmp, threads=os.cpu_count() or 8)[0]
                meta[name] = {k: r[k] for k in ("iterations", "phase", "primal_obj", "dual_obj",
                                                "seconds")}
                arrays[name + ".xvec"] = r["xvec"]
                print(name, meta[name], flush=True)
            r = run_ref([big[0][1]], tmp, param=tpath, threads=os.cpu_count() or 8)[0]
            meta["lt200.tight"] = {k: r[k] for k in ("iterations", "phase", "primal_obj", "dual_obj")}
            arrays["lt200.tight"] = r["xvec"]
            with open(os.path.join(HERE, "large.json"), "w") as f:
                json.dump(meta, f, indent=1)
            np.savez_compressed(os.path.join(HERE, "large.npz"), **arrays)


if __name__ == "__main__":
    main()
