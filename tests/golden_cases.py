"""Load the golden fixtures (tests/golden/*.npz) written by make_golden.py."""

import glob
import os
from types import SimpleNamespace

import numpy as np

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def names():
    return sorted(os.path.splitext(os.path.basename(p))[0]
                  for p in glob.glob(os.path.join(HERE, "*.npz")))


def load(name):
    """(problem, expected) for one case.  The problem is built with this
    repository's own Problem/SparseMatrix types from the stored CSC arrays."""
    from sovereign_moe_b200.problem import ObjSense, Problem, SparseMatrix
    d = np.load(os.path.join(HERE, f"{name}.npz"), allow_pickle=False)
    A = SparseMatrix(int(d["m"]), int(d["n"]), d["cp"], d["ci"], d["cx"])
    prob = Problem(A=A, c=d["c"], row_lb=d["row_lb"], row_ub=d["row_ub"],
                   col_lb=d["col_lb"], col_ub=d["col_ub"], kind=d["kind"],
                   obj_offset=float(d["obj_offset"]), sense=ObjSense(int(d["sense"])),
                   name=name)
    exp = SimpleNamespace(**{k: d[k] for k in d.files})
    return prob, exp


# parameters each case was solved with (make_golden.py)
PARAMS = {
    "toy": {}, "testprob": {}, "toy_min": {},
    **{f"badly_scaled_s{s}": dict(max_iter=60_000, time_limit=60) for s in range(4)},
    "dual_regression": dict(max_iter=60_000, time_limit=60),
    "agree": dict(eps_abs=1e-7, eps_rel=1e-7, max_iter=20_000),
    "randlp_2000": dict(eps_abs=1e-6, eps_rel=1e-6, max_iter=5000, time_limit=180),
    "small_known_s0": dict(eps_abs=1e-6, eps_rel=1e-6),
    "small_known_s1": dict(eps_abs=1e-6, eps_rel=1e-6),
    "small_known_iterlimit": dict(eps_abs=1e-6, eps_rel=1e-6, max_iter=100),
    "blend_mini": dict(eps_abs=1e-6, eps_rel=1e-6, max_iter=60_000, time_limit=300),
}
