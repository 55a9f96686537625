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


def rel(a, b):
    return abs(a - b) / max(1.0, abs(b))
