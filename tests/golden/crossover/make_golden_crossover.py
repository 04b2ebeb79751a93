"""Generate the golden fixtures that pin the crossover to the reference.

Runs the reference ``sovopt`` itself (imported read-only from a checkout of
manabsen006-a11y/Sovereign-MOE) and stores, per case and per starting point:
the status vector its ``basis_from_point`` identifies (as its ``crossover``
calls it, on the minimising form), what its ``crossover`` returns (status,
objective, pivots) and what a cold ``solve_simplex`` returns (status,
objective, pivots).  ``tests/test_crossover_cpu.py`` replays them.

Usage (needs the reference checkout; not run by the tests):

    SOVOPT_JIT_CACHE=0 PYTHONDONTWRITEBYTECODE=1 \\
        python tests/golden/crossover/make_golden_crossover.py /path/to/Sovereign-MOE

The cases: the LPs of the reference's crossover tests (``random_lp`` of its
simplex tests, seeds 0-4, from its interior-point and PDLP points; the
two-row LP with a pinned column; the maximising toy LP), and every LP of
``tests/golden/`` from the reference PDLP point stored there.
"""

from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.dirname(HERE)


def main(ref_root):
    os.environ.setdefault("SOVOPT_JIT_CACHE", "0")
    sys.dont_write_bytecode = True
    sys.path.insert(0, os.path.join(ref_root, "src"))
    sys.path.insert(0, ref_root)

    from sovopt.core.problem import ObjSense, Problem as RProblem
    from sovopt.core.sparse import SparseMatrix as RSparse
    from sovopt.core.tolerances import INF
    from sovopt.lp.crossover import basis_from_point, crossover
    from sovopt.lp.ipm import IPMParams, solve_ipm
    from sovopt.lp.pdlp import PDLPParams, solve_pdlp
    from sovopt.lp.simplex import SimplexParams, solve_simplex

    sys.path.insert(0, os.path.join(ref_root, "tests"))
    import test_simplex as tsx                               # tests/test_simplex.py

    def from_npz(z):
        A = RSparse(int(z["m"]), int(z["n"]), z["cp"], z["ci"], z["cx"])
        return RProblem(A=A, c=z["c"], row_lb=z["row_lb"], row_ub=z["row_ub"],
                        col_lb=z["col_lb"], col_ub=z["col_ub"],
                        sense=ObjSense(int(z["sense"])), obj_offset=float(z["obj_offset"]))

    def pinned_lp():
        # the two-row LP of the reference's "a fixed variable is never made
        # basic" test: column 1 has equal bounds
        A = RSparse.from_dense(np.array([[1., 1., 1.], [1., -1., 0.]]))
        return RProblem(A=A, c=np.array([1., 1., -1.]),
                        row_lb=np.array([1.0, -INF]), row_ub=np.array([1.0, 3.0]),
                        col_lb=np.array([0.0, 2.0, 0.0]), col_ub=np.array([5.0, 2.0, 5.0]))

    def identified(p, x, y):
        # crossover.py:206-212: the minimising form and the negated duals
        work, yy = p, y
        if p.sense == ObjSense.MAXIMISE:
            work = p.copy()
            work.c = -work.c
            yy = -np.asarray(y)
        return basis_from_point(work, x, yy)

    cases = []      # (name, problem, base golden or None, {point: (x, y)})
    for s in range(5):
        p = tsx.random_lp(seed=s)
        ip = solve_ipm(p.copy(), IPMParams())
        fo = solve_pdlp(p.copy(), PDLPParams(device="cpu", eps_abs=1e-8, eps_rel=1e-8))
        cases.append((f"random_lp_s{s}", p, None,
                      {"ipm": (ip.x, ip.y), "pdlp": (fo.x, fo.y)}))
    p = pinned_lp()
    ip = solve_ipm(p.copy(), IPMParams())
    cases.append(("pinned", p, None, {"ipm": (ip.x, ip.y)}))
    p = tsx.toy_lp()
    ip = solve_ipm(p.copy(), IPMParams())
    cases.append(("toy_max", p, None, {"ipm": (ip.x, ip.y)}))
    with open(os.path.join(GOLDEN, "manifest.json")) as fh:
        names = [c["name"] for c in json.load(fh)]
    for name in names:
        z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
        cases.append((name, from_npz(z), name, {"pdlp": (z["x"], z["y"])}))

    manifest = []
    for name, p, base, points in cases:
        cold = solve_simplex(p.copy(), SimplexParams())
        rec = dict(cold_status=int(cold.status), cold_objective=float(cold.objective),
                   cold_iterations=int(cold.iterations))
        if base is None:
            A = p.A
            rec.update(m=A.m, n=A.n, cp=A.cp, ci=A.ci, cx=A.cx, c=p.c,
                       row_lb=p.row_lb, row_ub=p.row_ub, col_lb=p.col_lb, col_ub=p.col_ub,
                       obj_offset=p.obj_offset, sense=int(p.sense))
        else:
            rec["base"] = base
        entry = dict(name=name, base=base, cold=[int(cold.status), float(cold.objective),
                                                 int(cold.iterations)], points={})
        for kind, (x, y) in points.items():
            st = identified(p, x, y)
            xo = crossover(p.copy(), x, y)
            if base is None:
                rec[f"{kind}_x"] = np.asarray(x)
                rec[f"{kind}_y"] = np.asarray(y)
            rec[f"{kind}_status"] = st
            rec[f"{kind}_xo_status"] = int(xo.status)
            rec[f"{kind}_xo_objective"] = float(xo.objective)
            rec[f"{kind}_xo_iterations"] = int(xo.iterations)
            rec[f"{kind}_xo_basis"] = xo.basis_status
            entry["points"][kind] = [int(xo.status), float(xo.objective), int(xo.iterations)]
            print(f"{name:22s} {kind:5s} cold {cold.status.name} {cold.objective:.12g} "
                  f"({cold.iterations} pivots)  crossover {xo.status.name} "
                  f"{xo.objective:.12g} ({xo.iterations} pivots)")
        rec["points"] = np.array(list(points))
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **rec)
        manifest.append(entry)
    with open(os.path.join(HERE, "manifest.json"), "w") as fh:
        json.dump(manifest, fh, indent=1)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden_crossover.py REFERENCE_ROOT")
    main(sys.argv[1])
