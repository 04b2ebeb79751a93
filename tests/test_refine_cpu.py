"""Host-side pieces of the mixed-precision path (no GPU): the equality form
with slack columns that the refinement rounds solve, checked with the CPU
oracle -- the same optimum, and the slack duals carry the row prices."""

import numpy as np

import golden_cases as gc
from oracle import pdlp_oracle as po
from sovereign_moe_b200.problem import Problem, SparseMatrix
from sovereign_moe_b200.refine import equality_form


def test_equality_form_keeps_the_optimum():
    prob, exp = gc.load("toy")                         # max 3x + 2y, three <= rows
    A2, c2, b, lo, hi, n0, flip = equality_form(prob)
    assert flip and n0 == 2 and A2.n == 2 + 3 and A2.m == 3
    eq = Problem(A=A2, c=c2, row_lb=b, row_ub=b, col_lb=lo, col_ub=hi)
    s = po.solve_pdlp(eq, dict(eps_abs=1e-9, eps_rel=1e-9))
    assert s.status == po.OPTIMAL
    assert abs(-s.objective - 11.0) < 1e-7              # min of -c
    assert np.allclose(s.x[:2], [3.0, 1.0], atol=1e-6)


def test_equality_rows_need_no_slacks():
    prob, _ = gc.load("small_known_s0")
    A2, c2, b, lo, hi, n0, flip = equality_form(prob)
    assert A2 is prob.A and not flip and n0 == prob.n
    np.testing.assert_array_equal(b, prob.row_lb)


def test_one_refinement_round_closes_the_gap():
    """Float64 residual LP solved loosely (1e-4) and added back: the primal
    violation and the gap drop by orders of magnitude (the arithmetic of
    sovereign_moe_b200.refine, with the CPU oracle as the inner solver)."""
    prob, _ = gc.load("small_known_s1")
    A = prob.A
    inner = dict(eps_abs=1e-4, eps_rel=1e-4, feas_cap=1e300)
    s = po.solve_pdlp(prob, inner)
    x, y = s.x, s.y
    res0 = np.abs(prob.row_lb - A.matvec(x)).max()
    dbar = prob.c - A.rmatvec(y)
    dp = dd = 1.0 / res0
    R = Problem(A=A, c=dd * dbar, row_lb=dp * (prob.row_lb - A.matvec(x)),
                row_ub=dp * (prob.row_lb - A.matvec(x)),
                col_lb=dp * (prob.col_lb - x), col_ub=dp * (prob.col_ub - x))
    r = po.solve_pdlp(R, inner)
    x2 = x + r.x / dp
    res1 = np.abs(prob.row_lb - A.matvec(x2)).max()
    assert res1 < 1e-3 * res0
