"""Loads the golden fixtures of tests/golden (made by tests/golden/make_golden.py
from the reference solver's own output)."""
import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def small():
    meta = json.load(open(os.path.join(GOLDEN, "small.json")))
    arr = np.load(os.path.join(GOLDEN, "small.npz"))
    return meta, arr


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


def x_within_reference_accuracy(x, x_ref, x_tight, tol=1e-5):
    """Parity bar on x for paths that leave the reference's iterate sequence
    (warm start, mixed precision).  At the default stopping test the
    reference's own x is determined only to |x_ref - x*| (x* its solution at
    epsilonStar 1e-11; up to 1.5e-4 on batched MaxCut, more where the optimal
    face is not a point), so such a path must land at least as close to x*
    as the reference does, up to `tol`."""
    return float(np.max(np.abs(x - x_tight))) <= float(np.max(np.abs(x_ref - x_tight))) + tol


def rel(a, b):
    return abs(a - b) / max(1.0, abs(b))
