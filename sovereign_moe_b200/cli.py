"""Command line: ``python -m sovereign_moe_b200 solve MODEL.mps [options]``.

The ``solve`` subcommand follows ``sovopt solve --method pdlp`` (the
reference's ``src/sovopt/cli.py:163-166, 234-313``): it reads an MPS model,
solves it with ``solve_pdlp`` at ``eps_abs = eps_rel = --tol`` on the GPU,
prints the same report (status, objective, iterations, method, time, row and
bound violation), and with ``--out`` writes the same JSON payload:
``model``, ``status``, ``objective``, ``dual_bound``, ``time``, ``method``,
``x`` and ``y`` (lists, or name-keyed objects with ``--named``).  That file
is what the reference's verifier (``bench/verify.py:279-318``) reads.

``--crossover`` crosses the PDLP point over to an optimal basis
(``crossover.py``; the reference's ``cli.py:167-182`` with the parameters it
passes: feas_tol = opt_tol = max(tol, 1e-9)).  In the reference the
``--method pdlp`` branch returns before the crossover branch is reached
(``cli.py:163-166``), so there the flag takes effect only with ``--method
ipm``; here it applies to the PDLP solve.

Extensions of this build: ``--precision fp32`` (float32 sparse products) and
``--refine`` (float32 inner solves with float64 iterative refinement to
``--tol``).  Only ``--method pdlp`` exists here; the reference's other
engines are out of scope.
"""

from __future__ import annotations

import argparse
import json
import sys
import time

import numpy as np

from .problem import ObjSense, Status

__all__ = ["main"]


def _stats(prob):
    A = prob.A
    rl, ru = np.asarray(prob.row_lb), np.asarray(prob.row_ub)
    from .problem import INF
    lo_f, hi_f = rl > -INF, ru < INF
    eq = int(np.sum(lo_f & hi_f & (rl == ru)))
    rng = int(np.sum(lo_f & hi_f & (rl != ru)))
    le = int(np.sum(~lo_f & hi_f))
    ge = int(np.sum(lo_f & ~hi_f))
    free = int(np.sum(~lo_f & ~hi_f))
    ints = int(np.count_nonzero(prob.kind)) if prob.kind is not None else 0
    ax = np.abs(np.asarray(A.cx))
    ax = ax[ax > 0]
    amin = float(ax.min()) if ax.size else 0.0
    amax = float(ax.max()) if ax.size else 0.0
    dens = A.nnz / max(1, A.m * A.n)
    return (f"{prob.name}  [{'MILP' if ints else 'LP'}]\n"
            f"  {A.m:,} rows x {A.n:,} cols, {A.nnz:,} nonzeros (density {dens:.2e})\n"
            f"  rows: {eq:,} eq, {le:,} <=, {ge:,} >=, {rng:,} ranged, {free:,} free\n"
            f"  cols: {A.n - ints:,} continuous, {ints:,} integer\n"
            f"  |a_ij| in [{amin:.3e}, {amax:.3e}]  ratio {amax / amin if amin else 0.0:.2e}")


def cmd_solve(a) -> int:
    from .mps import read_mps
    from .pdlp import PDLPParams, solve_pdlp
    prob = read_mps(a.model)
    if a.maximise:
        prob.sense = ObjSense.MAXIMISE
    if prob.kind is not None and np.any(prob.kind):
        print("  note: integrality is ignored; PDLP solves the LP relaxation")
    print(_stats(prob))
    print()
    params = PDLPParams(device=a.device, eps_abs=a.tol, eps_rel=a.tol,
                        time_limit=a.time_limit, verbose=a.verbose, precision=a.precision)
    t = time.perf_counter()
    if a.refine:
        from .refine import solve_refined
        sol = solve_refined(prob, params, target=a.tol)
    else:
        sol = solve_pdlp(prob, params)
    if a.crossover and sol.x is not None:
        from .crossover import crossover
        from .simplex import SimplexParams
        sol = crossover(prob, sol.x, sol.y,
                        SimplexParams(time_limit=a.time_limit, feas_tol=max(a.tol, 1e-9),
                                      opt_tol=max(a.tol, 1e-9), verbose=a.verbose))
    dt = time.perf_counter() - t
    print()
    print(f"  status      {sol.status.name}")
    if np.isfinite(sol.objective):
        print(f"  objective   {sol.objective:.12g}")
    if sol.iterations:
        print(f"  iterations  {sol.iterations:,}")
    print(f"  method      {sol.method}")
    print(f"  time        {dt:.3f}s")
    if sol.x is not None:
        rv, bv, iv = prob.violation(sol.x)
        print(f"  violation   row {rv:.2e}  bound {bv:.2e}  integrality {iv:.2e}")
    if a.out and sol.x is not None:
        cn = prob.col_names or [f"C{i}" for i in range(prob.n)]
        rn = prob.row_names or [f"R{i}" for i in range(prob.m)]
        payload = {
            "model": prob.name,
            "status": sol.status.name,
            "objective": sol.objective if np.isfinite(sol.objective) else None,
            "dual_bound": sol.dual_bound if np.isfinite(sol.dual_bound) else None,
            "time": dt,
            "method": sol.method,
            "x": ({n: float(v) for n, v in zip(cn, sol.x)} if a.named
                  else [float(v) for v in sol.x]),
        }
        if sol.y is not None and len(sol.y) == prob.m:
            payload["y"] = ({n: float(v) for n, v in zip(rn, sol.y)} if a.named
                            else [float(v) for v in sol.y])
        with open(a.out, "w", encoding="utf-8") as fh:
            json.dump(payload, fh, indent=1)
        print(f"  wrote       {a.out}")
    if a.print_solution and sol.x is not None:
        names = prob.col_names or [f"C{i}" for i in range(prob.n)]
        nz = np.flatnonzero(np.abs(sol.x) > 1e-9)
        print(f"\n  nonzero variables ({len(nz)} of {prob.n}):")
        for j in nz[:a.print_solution]:
            print(f"    {names[j]:<24s} {sol.x[j]:.10g}")
        if len(nz) > a.print_solution:
            print(f"    ... {len(nz) - a.print_solution} more")
    return 0 if sol.status == Status.OPTIMAL else 1


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(prog="python -m sovereign_moe_b200",
                                 description="B200 PDLP engine")
    sub = ap.add_subparsers(dest="cmd", required=True)
    p = sub.add_parser("solve", help="solve an MPS model with PDLP on the GPU")
    p.add_argument("model")
    p.add_argument("--method", choices=["pdlp"], default="pdlp")
    p.add_argument("--device", choices=["auto", "gpu"], default="auto")
    p.add_argument("--time-limit", type=float, default=300.0)
    p.add_argument("--tol", type=float, default=1e-8, help="LP tolerance (eps_abs = eps_rel)")
    p.add_argument("--maximise", action="store_true")
    p.add_argument("--out", help="write the solution as JSON")
    p.add_argument("--named", action="store_true",
                   help="key x and y by column and row names in the JSON")
    p.add_argument("--print-solution", type=int, default=0, metavar="N")
    p.add_argument("--precision", choices=["fp64", "fp32"], default="fp64")
    p.add_argument("--crossover", action="store_true",
                   help="cross the PDLP point over to an optimal simplex basis")
    p.add_argument("--refine", action="store_true",
                   help="float32 inner solves, float64 iterative refinement to --tol")
    p.add_argument("-v", "--verbose", action="store_true")
    p.set_defaults(fn=cmd_solve)
    a = ap.parse_args(argv)
    return a.fn(a)


if __name__ == "__main__":
    sys.exit(main())
