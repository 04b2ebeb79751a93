"""The revised simplex that finishes a crossover (sovopt ``lp/simplex.py``).

``solve_simplex(prob, params=None, warm_basis=None) -> Solution`` has the
reference's signature and result fields (``src/sovopt/lp/simplex.py:
1181-1374``): the primal point, row duals, reduced costs and the final basis
status vector, so the result can warm-start a later solve or answer a
ranging question.  It runs ``pdlp_simplex_solve`` of the C library on the
host cores: a bounded primal simplex over ``[A | -I]`` with a sparse LU of
the basis and product-form updates (``csrc/crossover.cu``).

What is the same as the reference: the computational form, the status
codes, the warm start from a status vector with exactly m basic entries
(else the all-logical basis with nonbasics at the bound their cost prefers),
the tolerances' names and defaults, the sign handling of a maximisation and
the checks on the returned point (``simplex.py:1309-1347``: x clipped to its
bounds; a point that violates the model by more than max(feas_tol, 1e-6)
makes an OPTIMAL status NUMERICAL and is dropped under a limit status).
What is not: the reference chooses between a dual and a two-phase primal
simplex and prices with devex, perturbs costs and scales the model; this one
always runs the composite two-phase primal with Dantzig pricing, on the
model as given.  Both end only at an optimal basis, so objectives agree to
the tolerances; pivot counts differ, and so may the basis of a degenerate LP.
"""

from __future__ import annotations

import ctypes
import time
from dataclasses import dataclass

import numpy as np

from . import _lib
from .pdlp import _result_types, problem_desc
from .problem import ObjSense


@dataclass
class SimplexParams:
    """The fields of sovopt's ``SimplexParams`` (simplex.py:94-196) this
    simplex uses, with the same defaults.  The reference's own
    ``SimplexParams`` is accepted too (read by attribute)."""

    max_iter: int = 1_000_000
    time_limit: float = 300.0
    feas_tol: float = 1e-7
    opt_tol: float = 1e-7
    pivot_tol: float = 1e-7
    refactor_freq: int = 150
    sensitivity: bool = False
    verbose: bool = False


def params_struct(params) -> _lib.SimplexParamsC:
    p = params if params is not None else SimplexParams()
    d = SimplexParams()
    s = _lib.SimplexParamsC()
    s.feas_tol = float(getattr(p, "feas_tol", d.feas_tol))
    s.opt_tol = float(getattr(p, "opt_tol", d.opt_tol))
    s.pivot_tol = float(getattr(p, "pivot_tol", d.pivot_tol))
    s.max_iter = int(getattr(p, "max_iter", d.max_iter))
    s.time_limit = float(getattr(p, "time_limit", d.time_limit))
    s.refactor_freq = int(getattr(p, "refactor_freq", d.refactor_freq))
    return s


def minimising_desc(prob):
    """``problem_desc`` of ``prob`` with c negated for a maximisation (the C
    simplex minimises).  Returns ``(desc, keepalive, flip)``."""
    desc, keep = problem_desc(prob)
    flip = int(prob.sense) == int(ObjSense.MAXIMISE)
    if flip:
        keep["c_min"] = np.ascontiguousarray(-np.asarray(prob.c, dtype=np.float64))
        desc.c = keep["c_min"].ctypes.data if keep["c_min"].size else None
    return desc, keep, flip


def solve_simplex(prob, params=None, warm_basis=None):
    """Solve an LP to an optimal basis (simplex.py:1181-1374)."""
    params = params if params is not None else SimplexParams()
    if getattr(prob, "Q", None) is not None:
        raise NotImplementedError("solve_simplex optimises a linear objective; this model "
                                  "has a quadratic term")
    sol_cls, st_cls, _ = _result_types(prob, None)
    t0 = time.perf_counter()
    lib = _lib.load()
    m, n = int(prob.A.m), int(prob.A.n)
    desc, keep, flip = minimising_desc(prob)
    warm = None
    if warm_basis is not None and len(warm_basis) == n + m:
        warm = np.ascontiguousarray(warm_basis, dtype=np.uint8)
    x = np.zeros(n)
    y = np.zeros(m)
    d = np.zeros(n)
    basis = np.zeros(n + m, dtype=np.uint8)
    info = _lib.SimplexInfo()
    _lib.check(lib.pdlp_simplex_solve(ctypes.byref(desc), ctypes.byref(params_struct(params)),
                                      warm.ctypes.data if warm is not None else None,
                                      x.ctypes.data, y.ctypes.data, d.ctypes.data,
                                      basis.ctypes.data, ctypes.byref(info)))
    del keep
    status = st_cls(int(info.status))
    x = np.clip(x, prob.col_lb, prob.col_ub)
    obj = float(np.asarray(prob.c) @ x) + float(prob.obj_offset)
    if flip:
        y, d = -y, -d
    feas_tol = float(getattr(params, "feas_tol", 1e-7))
    worst = None
    if status.has_solution and status != st_cls.OPTIMAL:
        row_v, col_v, _ = prob.violation(x)
        if max(row_v, col_v) > max(feas_tol, 1e-6):
            x, obj = None, float("nan")
    elif status == st_cls.OPTIMAL:
        row_v, col_v, _ = prob.violation(x)
        worst = max(row_v, col_v)
        if worst > max(feas_tol, 1e-6):
            status = st_cls.NUMERICAL
    sol = sol_cls(status=status, x=x, objective=obj, y=y, reduced_costs=d,
                  basis_status=basis, iterations=int(info.iterations),
                  time=time.perf_counter() - t0, method="simplex[primal]")
    sol.dual_bound = obj
    sol.info = {"factorizations": int(info.factorizations), "repairs": int(info.repairs),
                "phase1_iterations": int(info.phase1_iterations),
                "bound_flips": int(info.bound_flips),
                "degenerate_pivots": int(info.degenerate_pivots),
                "dual_iterations": int(info.dual_iterations),
                "cost_shifts": int(info.cost_shifts),
                "lu_nnz": int(info.lu_nnz), "algorithm": "primal",
                "primal_infeasibility": float(info.primal_infeasibility),
                "dual_infeasibility": float(info.dual_infeasibility),
                "native_seconds": float(info.seconds)}
    if worst is not None:
        sol.info["worst_violation"] = worst
    return sol.drop_objective_if_unsolved()
