"""Generate the golden fixtures that pin the CPU oracle to the reference.

Runs the reference ``sovopt`` itself (imported read-only from a checkout of
manabsen006-a11y/Sovereign-MOE) on a set of LPs and stores, per case, the
problem arrays, the parameters, and what the reference returned: status,
iteration / restart / rejected-step counts, objective, x, y, reduced costs,
final step size and primal weight, the check history, the ``method="pdlp"``
scale factors, and the verifier's verdict.  ``tests/test_oracle_golden.py``
replays every case through ``oracle/`` and demands the same outputs.

Usage (needs the reference checkout; not run by the tests):

    SOVOPT_JIT_CACHE=0 PYTHONDONTWRITEBYTECODE=1 \
        python tests/golden/make_golden.py /path/to/Sovereign-MOE

The problems: the reference's own PDLP known-answer LPs (the toy LP with
optimum 11, the MPS fixture with optimum 16, the badly scaled family of its
solver tests, the random LP of its GPU agreement test and of its GPU bench),
plus known-optimum LPs of this repository's workload generators.
"""

from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))


def main(ref_root):
    os.environ.setdefault("SOVOPT_JIT_CACHE", "0")
    sys.dont_write_bytecode = True
    sys.path.insert(0, os.path.join(ref_root, "src"))
    sys.path.insert(0, ref_root)
    sys.path.insert(0, REPO)

    from sovopt.core.problem import ObjSense, Problem as RProblem
    from sovopt.core.sparse import SparseMatrix as RSparse
    from sovopt.core.tolerances import INF
    from sovopt.io.mps import read_mps
    from sovopt.lp.pdlp import PDLPParams, solve_pdlp
    from sovopt.numerics.scaling import scale_problem
    from bench.verify import verify
    from bench.gpu_bench import make_lp
    from sovereign_moe_b200 import workloads

    sys.path.insert(0, os.path.join(ref_root, "tests"))
    import test_solvers as ts                              # tests/test_solvers.py

    def to_ref(p):
        A = RSparse(p.A.m, p.A.n, p.A.cp, p.A.ci, p.A.cx)
        return RProblem(A=A, c=p.c, row_lb=p.row_lb, row_ub=p.row_ub,
                        col_lb=p.col_lb, col_ub=p.col_ub, sense=p.sense,
                        obj_offset=p.obj_offset, name=p.name)

    def agree_lp():
        # the LP of the reference GPU agreement test: 300 x 400, 5 entries
        # per column, one-sided rows around a random interior point
        rng = np.random.default_rng(11)
        m, n = 300, 400
        sub = np.random.default_rng(11)
        cols = np.repeat(np.arange(n), 5)
        rows = sub.integers(0, m, cols.size)
        vals = sub.standard_normal(cols.size)
        A = RSparse.from_triplets(rows, cols, vals, m, n)
        b = A.matvec(rng.random(n)) + rng.random(m) * 0.5
        return RProblem(A=A, c=rng.standard_normal(n), row_lb=np.full(m, -INF),
                        row_ub=b, col_lb=np.zeros(n), col_ub=np.full(n, 10.0),
                        name="agree")

    cases = []
    cases.append(("toy", ts.toy_lp(), {}, 11.0))
    cases.append(("testprob", read_mps(os.path.join(ref_root, "tests", "fixtures",
                                                     "testprob.mps")), {}, 16.0))
    toy_min = ts.toy_lp().copy()
    toy_min.c = -toy_min.c
    toy_min.sense = ObjSense.MINIMISE
    cases.append(("toy_min", toy_min, {}, -11.0))
    for s in range(4):
        cases.append((f"badly_scaled_s{s}", ts.badly_scaled_lp(seed=s),
                      dict(max_iter=60_000, time_limit=60), None))
    cases.append(("dual_regression", ts.badly_scaled_lp(seed=1, m=30, n=40, spread=4),
                  dict(max_iter=60_000, time_limit=60), None))
    cases.append(("agree", agree_lp(), dict(eps_abs=1e-7, eps_rel=1e-7, max_iter=20_000), None))
    cases.append(("randlp_2000", make_lp(2000, 3000, 6, seed=2000),
                  dict(eps_abs=1e-6, eps_rel=1e-6, max_iter=5000, time_limit=180), None))
    for s in (0, 1):
        k = workloads.single_small(seed=s)
        cases.append((f"small_known_s{s}", to_ref(k.problem),
                      dict(eps_abs=1e-6, eps_rel=1e-6), k.f_star))
    k = workloads.single_small(seed=2)
    cases.append(("small_known_iterlimit", to_ref(k.problem),
                  dict(eps_abs=1e-6, eps_rel=1e-6, max_iter=100), None))
    k = workloads.blending_plan(seed=0, m=1200, n=3600, periods=6, coupling=10)
    cases.append(("blend_mini", to_ref(k.problem),
                  dict(eps_abs=1e-6, eps_rel=1e-6, max_iter=60_000, time_limit=300), k.f_star))

    manifest = []
    for name, prob, kw, known in cases:
        params = PDLPParams(device="cpu", **kw)
        sol = solve_pdlp(prob, params)
        _, sc = scale_problem(prob, method="pdlp")
        v = verify(prob, sol.x, sol.objective if np.isfinite(sol.objective) else None,
                   feas_tol=1e-6, y=sol.y)
        A = prob.A
        hist = np.array(sol.log, dtype=np.float64).reshape(-1, 5)
        info = sol.info
        np.savez_compressed(
            os.path.join(HERE, f"{name}.npz"),
            m=A.m, n=A.n, cp=A.cp, ci=A.ci, cx=A.cx,
            c=prob.c, row_lb=prob.row_lb, row_ub=prob.row_ub,
            col_lb=prob.col_lb, col_ub=prob.col_ub,
            obj_offset=prob.obj_offset, sense=int(prob.sense),
            kind=prob.kind,
            status=int(sol.status), iterations=sol.iterations,
            restarts=info.restarts, rejected=info.rejected_steps,
            objective=sol.objective, x=sol.x, y=sol.y, reduced_costs=sol.reduced_costs,
            step_size=info.step_size, primal_weight=info.primal_weight,
            info_res=np.array([info.primal_res, info.dual_res, info.gap,
                               info.primal_obj, info.dual_obj]),
            history=hist, scale_row=sc.row, scale_col=sc.col, scale_obj=sc.obj,
            verify_ok=v.ok, verify_checks=np.array([c[1] for c in v.checks]),
            verify_names=np.array([c[0] for c in v.checks]),
            certified_bound=np.nan if v.certified_bound is None else v.certified_bound,
            known=np.nan if known is None else known,
        )
        manifest.append(dict(name=name, params=kw, status=sol.status.name,
                             iterations=sol.iterations, objective=sol.objective,
                             verify_ok=v.ok, known=known))
        print(f"{name:24s} {sol.status.name:16s} it={sol.iterations:6d} "
              f"obj={sol.objective:.12g} verify={v.ok}")
    with open(os.path.join(HERE, "manifest.json"), "w") as fh:
        json.dump(manifest, fh, indent=1)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {os.path.basename(__file__)} REFERENCE_ROOT  "
                 "(the root of the reference source tree, holding src/sovopt)")
    main(sys.argv[1])
