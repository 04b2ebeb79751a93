"""Crossover from a PDLP point to an optimal basis (sovopt ``lp/crossover.py``).

PDLP stops at a point that is optimal to a tolerance but not a vertex: it
has no basis, so no ranging and no warm start.  ``crossover(prob, x, y)``
turns the engine's point into an exact optimal basic solution in two steps,
the reference's (``src/sovopt/lp/crossover.py:1-222``):

1. ``basis_from_point`` scores every variable of ``[x ; s]`` by how far it
   sits from its nearest bound relative to its range, and pushes the
   candidates into the all-logical basis one FTRAN each, pivoting on the
   largest entry in a row that still holds its logical -- so the basis is
   nonsingular by construction (``pdlp_basis_from_point``; the same scores,
   order, pivot rule and statuses as ``crossover.py:80-187``).
2. ``solve_simplex`` finishes from that basis (``simplex.py`` here).

Both run on the host cores (pivoting is sequential); the point comes from
the device solve.  Returns the simplex's ``Solution`` with
``info["crossover"] = True``, ``info["crossover_time"]`` and the
identification's counts.
"""

from __future__ import annotations

import ctypes
import time

import numpy as np

from . import _lib
from .problem import ObjSense
from .simplex import SimplexParams, minimising_desc, solve_simplex

__all__ = ["basis_from_point", "crossover"]


def _identify(prob, x, y, params, tol_fixed, minimise):
    lib = _lib.load()
    m, n = int(prob.A.m), int(prob.A.n)
    if minimise:
        desc, keep, _ = minimising_desc(prob)
    else:
        from .pdlp import problem_desc
        desc, keep = problem_desc(prob)
    xx = np.ascontiguousarray(x, dtype=np.float64)
    if xx.shape != (n,):
        raise ValueError(f"x has shape {xx.shape}, expected ({n},)")
    yy = None
    if y is not None:
        yy = np.ascontiguousarray(y, dtype=np.float64)
        if yy.shape != (m,):
            raise ValueError(f"y has shape {yy.shape}, expected ({m},)")
    pivot_tol = max(float(getattr(params, "pivot_tol", 1e-7)), 1e-7)    # crossover.py:164-165
    status = np.zeros(n + m, dtype=np.uint8)
    info = _lib.CrossoverInfo()
    _lib.check(lib.pdlp_basis_from_point(ctypes.byref(desc), xx.ctypes.data,
                                         yy.ctypes.data if yy is not None else None,
                                         float(tol_fixed), pivot_tol, status.ctypes.data,
                                         ctypes.byref(info)))
    del keep
    return status, info


def basis_from_point(prob, x, y=None, params=None, tol_fixed: float = 1e-12):
    """Identify a candidate basis from a primal point, as a status vector of
    length n + m with exactly m ``BASIC`` entries (crossover.py:80-187).
    ``prob.c`` is taken as the cost to minimise, as in the reference (its
    ``crossover`` passes the negated cost of a maximisation)."""
    status, _ = _identify(prob, x, y, params if params is not None else SimplexParams(),
                          tol_fixed, minimise=False)
    return status


def crossover(prob, x, y=None, params=None):
    """Cross over from a PDLP (or interior) point to an optimal basic
    solution (crossover.py:190-222).  ``x``, ``y`` are in the caller's sense
    and units, as ``solve_pdlp`` returns them."""
    params = params if params is not None else SimplexParams()
    t0 = time.perf_counter()
    yy = y
    if y is not None and int(prob.sense) == int(ObjSense.MAXIMISE):
        yy = -np.asarray(y, dtype=np.float64)
    status, info = _identify(prob, x, yy, params, 1e-12, minimise=True)
    sol = solve_simplex(prob, params, warm_basis=status)
    sol.info = dict(getattr(sol, "info", None) or {})
    sol.info["crossover"] = True
    sol.info["crossover_time"] = time.perf_counter() - t0
    sol.info["identified"] = {"placed": int(info.placed), "candidates": int(info.candidates),
                              "rejected": int(info.rejected), "repairs": int(info.repairs),
                              "seconds": float(info.seconds)}
    return sol
