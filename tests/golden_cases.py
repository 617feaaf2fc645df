"""Loader for the golden vectors in tests/golden/ (made by make_golden.py from
the reference's own CPU build)."""
from __future__ import annotations

import json
import os

import numpy as np

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


class Case(dict):
    def arr(self, name):
        return self["_arrays"][f"{self['id']}_{name}"]


def load():
    with open(os.path.join(HERE, "golden.json")) as f:
        meta = json.load(f)
    arrays = dict(np.load(os.path.join(HERE, "golden.npz")))
    cases = []
    for c in meta["cases"]:
        cc = Case(c)
        cc["_arrays"] = arrays
        cases.append(cc)
    meta["cases"] = cases
    return meta


def rel_err(a, b):
    """Normwise max |a-b| / max |b| (0 when both vanish)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.max(np.abs(b)) if b.size else 0.0
    num = np.max(np.abs(a - b)) if a.size else 0.0
    if den == 0.0:
        return float(num)
    return float(num / den)


def ref_elementwise_err(a, b):
    """The reference tests' metric: min(max abs, max rel) with
    rel = |a-b| / (1 + max(|a|,|b|)) (test_kronmult6_xbatched.cpp:522-523)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    d = np.abs(a - b)
    rel = d / (1.0 + np.maximum(np.abs(a), np.abs(b)))
    return float(min(d.max(initial=0.0), rel.max(initial=0.0)))
