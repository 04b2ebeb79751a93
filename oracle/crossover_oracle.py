"""CPU restatement of the reference's basis identification -- TEST INFRASTRUCTURE ONLY.

``basis_from_point`` follows ``src/sovopt/lp/crossover.py:80-187`` step by
step: the same scores over ``[x ; s]``, the same candidate order, the same
push into the all-logical basis with the pivot on the largest ``|B^-1 M_j|``
entry in a row that still holds its logical, the same statuses.  The basis
inverse is kept here as an explicit dense matrix, updated by the product-form
step after each pivot and recomputed by ``numpy.linalg.inv`` every 60 pivots
(the reference refactorises its sparse LU at the same cadence,
``lp/basis.py:137``), so it is for small LPs only.  The sums ``A x`` and
``A^T y`` go through ``oracle/sparse_ref.c`` in the reference's order.

Pinned by ``tests/test_crossover_cpu.py`` against status vectors that the
reference itself produced (``tests/golden/crossover/``).

``kkt_of_basis`` is the checker for a basic solution: it recomputes the
primal values, duals and reduced costs of a status vector from scratch with
dense linear algebra and reports the worst primal and dual infeasibility.
"""

from __future__ import annotations

import numpy as np

from . import pdlp_oracle as po

INF = po.INF
BASIC, AT_LOWER, AT_UPPER, FREE, FIXED = 0, 1, 2, 3, 4    # lp/basis.py:75-79


def _bounds(prob):
    lower = np.concatenate([prob.col_lb, prob.row_lb]).astype(np.float64)
    upper = np.concatenate([prob.col_ub, prob.row_ub]).astype(np.float64)
    return lower, upper


def _dense_M(prob):
    """M = [A | -I] as a dense matrix."""
    A = prob.A
    D = np.zeros((A.m, A.n))
    for j in range(A.n):
        s, e = int(A.cp[j]), int(A.cp[j + 1])
        D[A.ci[s:e], j] = A.cx[s:e]
    return np.hstack([D, -np.eye(A.m)])


def basis_from_point(prob, x, y=None, tol_fixed=1e-12, pivot_tol=1e-7):
    """Status vector of length n + m (crossover.py:80-187)."""
    A = prob.A
    m, n = A.m, A.n
    N = n + m
    x = np.asarray(x, dtype=np.float64)
    s = po.spmv(A.rp, A.ri, A.rx, x)                       # crossover.py:112
    z = np.concatenate([x, s])
    lower, upper = _bounds(prob)
    has_lo = lower > -INF
    has_hi = upper < INF
    fixed = has_lo & has_hi & (upper - lower <= tol_fixed * np.maximum(1.0, np.abs(lower)))
    free = ~has_lo & ~has_hi

    d = np.zeros(N)                                        # crossover.py:126-130
    if y is not None:
        y = np.asarray(y, dtype=np.float64)
        d[:n] = prob.c - po.spmv(A.cp, A.ci, A.cx, y)
        d[n:] = y

    span = np.where(has_lo & has_hi, upper - lower, 0.0)  # crossover.py:136-141
    scale = np.maximum(1.0, np.where(span > 0, span, np.abs(z)))
    with np.errstate(invalid="ignore"):
        dist_lo = np.where(has_lo, z - lower, np.inf)
        dist_hi = np.where(has_hi, upper - z, np.inf)
        interior = np.minimum(dist_lo, dist_hi) / scale
    interior[~np.isfinite(interior)] = np.inf
    score = interior - 1e-9 * np.abs(d)                    # crossover.py:145-147
    score[fixed] = -np.inf
    score[free] = np.inf

    live = np.flatnonzero((score[:n] > 1e-9) & np.isfinite(score[:n]))   # :157-160
    order = live[np.argsort(-score[live], kind="stable")]
    forced = np.flatnonzero(free[:n])
    order = np.concatenate([forced, order[~np.isin(order, forced)]])

    M = _dense_M(prob)
    basic = np.arange(n, N)
    Binv = -np.eye(m)                                      # the logical basis, -I
    taken = np.zeros(m, dtype=bool)
    placed = since = 0
    for j in order:                                        # crossover.py:168-180
        if placed == m:
            break
        alpha = Binv @ M[:, j]
        mag = np.where(taken, 0.0, np.abs(alpha))
        r = int(np.argmax(mag))
        if mag[r] <= pivot_tol:
            continue
        piv = alpha[r]
        row = Binv[r] / piv                                # E^-1 applied to B^-1
        Binv -= np.outer(alpha, row)
        Binv[r] = row
        basic[r] = j
        taken[r] = True
        placed += 1
        since += 1
        if since >= 60:
            Binv = np.linalg.inv(M[:, basic])
            since = 0

    with np.errstate(invalid="ignore"):                    # crossover.py:182-187
        at_lower = (np.abs(z - lower) <= np.abs(upper - z)) | ~has_hi
    status = np.where(at_lower & has_lo, AT_LOWER,
                      np.where(has_hi, AT_UPPER, FREE)).astype(np.uint8)
    status[fixed] = FIXED
    status[basic] = BASIC
    return status


def kkt_of_basis(prob, status, minimise_c=None):
    """Worst primal and dual infeasibility of the basic solution ``status``
    names, recomputed densely: z_N at its bounds, z_B = B^-1(-M_N z_N),
    y = B^-T c_B, d = c - M^T y.  ``minimise_c``: the cost minimised (the
    negated c of a maximisation); default ``prob.c``.  Returns
    ``(x, y, d, primal_inf, dual_inf)``."""
    A = prob.A
    m, n = A.m, A.n
    c = np.asarray(prob.c if minimise_c is None else minimise_c, dtype=np.float64)
    cost = np.concatenate([c, np.zeros(m)])
    lower, upper = _bounds(prob)
    M = _dense_M(prob)
    status = np.asarray(status)
    basic = np.flatnonzero(status == BASIC)
    assert basic.size == m, "not exactly m basic variables"
    z = np.zeros(n + m)
    z[status == AT_LOWER] = lower[status == AT_LOWER]
    z[status == FIXED] = lower[status == FIXED]
    z[status == AT_UPPER] = upper[status == AT_UPPER]
    Bm = M[:, basic]
    z[basic] = np.linalg.solve(Bm, -(M @ z))
    y = np.linalg.solve(Bm.T, cost[basic])
    d = cost - M.T @ y
    d[basic] = 0.0
    p_inf = float(max(np.maximum(lower - z, 0.0).max(initial=0.0),
                      np.maximum(z - upper, 0.0).max(initial=0.0)))
    viol = np.zeros(n + m)
    viol[status == AT_LOWER] = np.maximum(-d[status == AT_LOWER], 0.0)
    viol[status == AT_UPPER] = np.maximum(d[status == AT_UPPER], 0.0)
    viol[status == FREE] = np.abs(d[status == FREE])
    return z[:n], y, d[:n], p_inf, float(viol.max(initial=0.0))
