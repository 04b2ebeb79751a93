"""Load the crossover fixtures (tests/golden/crossover/*.npz) written by
make_golden_crossover.py: the problem (stored, or the tests/golden case it
names), each starting point, and what the reference returned from it."""

import json
import os
from types import SimpleNamespace

import numpy as np

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "crossover")
BASE = os.path.dirname(HERE)


def names():
    with open(os.path.join(HERE, "manifest.json")) as fh:
        return [e["name"] for e in json.load(fh)]


def load(name):
    """``(problem, points, expected)``: points maps "ipm" / "pdlp" to (x, y)."""
    from sovereign_moe_b200.problem import ObjSense, Problem, SparseMatrix
    z = np.load(os.path.join(HERE, f"{name}.npz"), allow_pickle=False)
    base = str(z["base"]) if "base" in z.files else None
    src = np.load(os.path.join(BASE, f"{base}.npz"), allow_pickle=False) if base else z
    A = SparseMatrix(int(src["m"]), int(src["n"]), src["cp"], src["ci"], src["cx"])
    prob = Problem(A=A, c=src["c"], row_lb=src["row_lb"], row_ub=src["row_ub"],
                   col_lb=src["col_lb"], col_ub=src["col_ub"],
                   obj_offset=float(src["obj_offset"]), sense=ObjSense(int(src["sense"])),
                   name=name)
    points = {}
    for k in (str(v) for v in z["points"]):
        if base is None:
            points[k] = (z[f"{k}_x"], z[f"{k}_y"])
        else:
            points[k] = (src["x"], src["y"])
    exp = SimpleNamespace(**{k: z[k] for k in z.files})
    return prob, points, exp


def minimising(prob, y):
    """The form the reference's crossover identifies on (crossover.py:206-212):
    c negated and y negated for a maximisation."""
    from sovereign_moe_b200.problem import ObjSense
    if int(prob.sense) != int(ObjSense.MAXIMISE):
        return prob, y
    work = prob.copy()
    work.c = -work.c
    return work, -np.asarray(y)
