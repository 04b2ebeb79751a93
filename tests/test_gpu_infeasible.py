"""Infeasibility detection (an addition of this engine; the reference's PDLP
runs an infeasible LP to its iteration or time limit).

With ``detect_infeasibility`` the change of the iterates between tests is
checked as a Farkas ray: a primal-infeasible LP must end INFEASIBLE and a
dual-infeasible (unbounded) LP INFEASIBLE_OR_UNBOUNDED, well before the
iteration limit.  On feasible LPs the test must never fire and must leave the
solve bitwise unchanged (it only reads the iterates).
"""

import numpy as np
import pytest

import golden_cases as gc
from sovereign_moe_b200 import workloads
from sovereign_moe_b200.pdlp import PDLPParams, solve_pdlp
from sovereign_moe_b200.problem import INF, Problem, SparseMatrix, Status

pytestmark = pytest.mark.gpu


def _lp(rows, cols, vals, m, n, c, rl, ru, lo, hi):
    A = SparseMatrix.from_triplets(np.array(rows), np.array(cols), np.array(vals, float), m, n)
    return Problem(A=A, c=np.array(c, float), row_lb=np.array(rl, float),
                   row_ub=np.array(ru, float), col_lb=np.array(lo, float),
                   col_ub=np.array(hi, float))


def _params(detect=True, **kw):
    return PDLPParams(device="gpu", eps_abs=1e-6, eps_rel=1e-6, max_iter=50_000,
                      detect_infeasibility=detect, **kw)


def test_primal_infeasible_is_detected(require_gpu):
    # x1 + x2 >= 3 and x1 + x2 <= 1 on [0, 10]^2
    p = _lp([0, 0, 1, 1], [0, 1, 0, 1], [1, 1, 1, 1], 2, 2, [1, 1],
            [3, -INF], [INF, 1], [0, 0], [10, 10])
    s = solve_pdlp(p, _params())
    assert s.status == Status.INFEASIBLE
    assert s.iterations < 50_000
    assert np.isnan(s.objective)
    off = solve_pdlp(p, _params(detect=False))
    assert off.status != Status.INFEASIBLE


def test_unbounded_is_detected(require_gpu):
    # min -x1 - x2, x1 - x2 = 0, x >= 0: unbounded along (1, 1)
    p = _lp([0, 0], [0, 1], [1, -1], 1, 2, [-1, -1], [0], [0], [0, 0], [INF, INF])
    s = solve_pdlp(p, _params())
    assert s.status == Status.INFEASIBLE_OR_UNBOUNDED
    assert s.iterations < 50_000


def test_conflicting_rows_in_a_larger_lp(require_gpu):
    """A config-1 LP with one equality row duplicated at another right-hand
    side: infeasible, with the certificate y = e_dup - e_row."""
    k = workloads.single_small(seed=2)
    A = k.problem.A
    r = 7
    rows = list(np.repeat(np.arange(A.m), np.diff(A.rp)))
    cols = list(A.ri)
    vals = list(A.rx)
    p0, p1 = int(A.rp[r]), int(A.rp[r + 1])
    rows += [A.m] * (p1 - p0)
    cols += list(A.ri[p0:p1])
    vals += list(A.rx[p0:p1])
    rl = np.append(k.problem.row_lb, k.problem.row_lb[r] + 1.0)
    ru = np.append(k.problem.row_ub, k.problem.row_ub[r] + 1.0)
    p = _lp(rows, cols, vals, A.m + 1, A.n, k.problem.c, rl, ru, k.problem.col_lb,
            k.problem.col_ub)
    s = solve_pdlp(p, _params())
    assert s.status == Status.INFEASIBLE


@pytest.mark.parametrize("name", ["toy", "testprob", "agree", "small_known_s0",
                                  "small_known_s1", "badly_scaled_s0", "dual_regression"])
def test_no_false_positive_and_no_change(require_gpu, name):
    prob, _ = gc.load(name)
    kw = gc.PARAMS[name]
    on = solve_pdlp(prob, PDLPParams(device="gpu", detect_infeasibility=True, **kw))
    off = solve_pdlp(prob, PDLPParams(device="gpu", **kw))
    assert on.status == off.status
    assert on.iterations == off.iterations
    assert np.array_equal(on.x, off.x) and np.array_equal(on.y, off.y)


def test_server_ends_an_infeasible_request(require_gpu):
    from sovereign_moe_b200.serving import Server
    bad = _lp([0, 0, 1, 1], [0, 1, 0, 1], [1, 1, 1, 1], 2, 2, [1, 1],
              [3, -INF], [INF, 1], [0, 0], [10, 10])
    good = workloads.single_small(seed=0)
    with Server(max_slots=4) as srv:
        done, _ = srv.serve([(0.0, bad), (0.0, good.problem)], realtime=False)
    assert done[0].solution.status == Status.INFEASIBLE
    assert done[1].solution.status == Status.OPTIMAL
    assert abs(done[1].solution.objective - good.f_star) <= 1e-6 * max(1.0, abs(good.f_star))
