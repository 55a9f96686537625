"""Loads the golden fixtures of tests/golden (made by tests/golden/make_golden.py
from the reference solver's own output)."""
import json
import os

import numpy as np

from oracle.ref_runner import x_within_reference_accuracy  # noqa: F401  (the parity bar on x)

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def small():
    meta = json.load(open(os.path.join(GOLDEN, "small.json")))
    arr = np.load(os.path.join(GOLDEN, "small.npz"))
    return meta, arr


def blocks():
    """Reference results of the batched multi-block instances blk0..blk31."""
    meta = json.load(open(os.path.join(GOLDEN, "blocks.json")))
    return meta, np.load(os.path.join(GOLDEN, "blocks.npz"))


def known_answers():
    return json.load(open(os.path.join(GOLDEN, "known_answers.json")))


def large():
    p = os.path.join(GOLDEN, "large.json")
    if not os.path.exists(p):
        return None, None
    return json.load(open(p)), np.load(os.path.join(GOLDEN, "large.npz"))


def tight():
    """Reference solutions at epsilonStar 1e-11 (name -> x) and the reference's
    default-parameter results of the warm-start held-out set."""
    meta = json.load(open(os.path.join(GOLDEN, "tight.json")))
    return meta, np.load(os.path.join(GOLDEN, "tight.npz"))


def rel(a, b):
    return abs(a - b) / max(1.0, abs(b))


_NUM = None


def normalize_result_line(line: str) -> str:
    """A result-file line with every number replaced by '#' (layout only)."""
    import re
    global _NUM
    if _NUM is None:
        _NUM = re.compile(r"[+-]?(\d+\.?\d*|\.\d+)([eE][+-]?\d+)?")
    return _NUM.sub("#", line.rstrip("\n"))


def parse_result(text: str) -> dict:
    """The parts of an SDPA result file a script reads: the iteration table,
    the last-iteration block, the DIMACS errors and xVec / xMat / yMat."""
    import re
    lines = text.splitlines()
    out = {"table": [], "info": {}, "dimacs": {}, "layout": []}
    num = re.compile(r"[+-]?(?:\d+\.?\d*|\.\d+)(?:[eE][+-]?\d+)?")
    for ln in lines:
        if ln.startswith("SDPA start at") or ln.startswith("SDPA end at"):
            continue
        out["layout"].append(normalize_result_line(ln))
    i = 0
    while i < len(lines):
        ln = lines[i]
        t = ln.split()
        if len(t) == 9 and t[0].isdigit() and "e" in t[1]:
            out["table"].append([float(x) for x in t])
        elif "=" in ln and ln.split("=")[0].strip() in ("phase.value", "Iteration", "mu", "relative gap", "gap",
                                                          "digits", "objValPrimal", "objValDual",
                                                          "p.feas.error", "d.feas.error"):
            k, v = ln.split("=", 1)
            out["info"][k.strip()] = v.strip()
        elif re.match(r"err\d = ", ln):
            out["dimacs"][ln[:4]] = float(num.findall(ln[6:])[0])
        elif ln.strip() in ("xVec =", "xMat =", "yMat ="):
            key = ln.strip()[:4]
            buf = []
            j = i + 1
            depth = 0
            while j < len(lines):
                buf.append(lines[j])
                depth += lines[j].count("{") - lines[j].count("}")
                j += 1
                if depth == 0:
                    break
            out[key] = [float(x) for x in num.findall("\n".join(buf))]
            i = j - 1
        i += 1
    return out
