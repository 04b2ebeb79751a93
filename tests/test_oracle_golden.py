"""The CPU oracle against outputs of the reference itself.

tests/golden/*.npz hold what the reference solve_pdlp (device="cpu"),
scale_problem(method="pdlp") and bench.verify.verify returned on each case
(tests/golden/make_golden.py).  The oracle must reproduce them exactly: the
same scale factors, the same iteration/restart/rejection counts, the same x
and y to the last bit, the same verifier verdicts.
"""

import numpy as np
import pytest

import golden_cases as gc
from oracle import pdlp_oracle as po
from oracle import verify_oracle as vo

CASES = gc.names()


@pytest.mark.parametrize("name", CASES)
def test_scaling_matches_reference(name):
    prob, exp = gc.load(name)
    flip = int(prob.sense) == -1
    work = prob.copy()
    if flip:
        work.c = -work.c
        work.obj_offset = -work.obj_offset
    _, sc = po.scale_problem(work, method="pdlp")
    _, sc_plain = po.scale_problem(prob, method="pdlp")
    assert np.array_equal(sc_plain.row, exp.scale_row)
    assert np.array_equal(sc_plain.col, exp.scale_col)
    assert sc_plain.obj == float(exp.scale_obj)
    assert np.array_equal(sc.row, exp.scale_row)


@pytest.mark.parametrize("name", CASES)
def test_solve_matches_reference_bitwise(name):
    prob, exp = gc.load(name)
    s = po.solve_pdlp(prob, gc.PARAMS[name])
    assert s.status == int(exp.status)
    assert s.iterations == int(exp.iterations)
    assert s.info.restarts == int(exp.restarts)
    assert s.info.rejected_steps == int(exp.rejected)
    assert np.array_equal(s.x, exp.x)
    assert np.array_equal(s.y, exp.y)
    assert np.array_equal(s.reduced_costs, exp.reduced_costs)
    if np.isfinite(exp.objective):
        assert s.objective == float(exp.objective)
    else:
        assert not np.isfinite(s.objective)
    assert s.info.step_size == float(exp.step_size)
    assert s.info.primal_weight == float(exp.primal_weight)
    hist = np.array(s.info.history, dtype=np.float64).reshape(-1, 5)
    assert np.array_equal(hist, exp.history)


@pytest.mark.parametrize("name", CASES)
def test_verifier_matches_reference(name):
    prob, exp = gc.load(name)
    claimed = float(exp.objective) if np.isfinite(exp.objective) else None
    v = vo.verify(prob, exp.x, claimed, feas_tol=1e-6, y=exp.y)
    assert v.ok == bool(exp.verify_ok)
    assert [c[0] for c in v.checks] == [str(s) for s in exp.verify_names]
    assert [c[1] for c in v.checks] == [bool(b) for b in exp.verify_checks]
    if np.isfinite(exp.certified_bound):
        assert v.certified_bound == pytest.approx(float(exp.certified_bound), rel=1e-12, abs=1e-12)


def test_known_answers():
    """The reference's own known-answer tests (tests/test_solvers.py:50-66)."""
    prob, _ = gc.load("toy")
    s = po.solve_pdlp(prob)
    assert s.status == po.OPTIMAL and abs(s.objective - 11.0) < 1e-6
    assert np.allclose(s.x, [3.0, 1.0], atol=1e-5)
    prob, _ = gc.load("testprob")
    s = po.solve_pdlp(prob)
    assert s.status == po.OPTIMAL and abs(s.objective - 16.0) < 1e-7
    assert np.allclose(s.x, [0.0, -1.0, 6.0], atol=1e-6)


def test_planted_mistake_is_caught():
    """A deliberately wrong oracle (objective scale multiplied instead of
    divided in the dual unscaling, the reference's regression of
    tests/test_solvers.py:69-99) must disagree with the golden duals."""
    prob, exp = gc.load("dual_regression")
    s = po.solve_pdlp(prob, gc.PARAMS["dual_regression"])
    sc = s.scaling
    wrong_y = s.y * sc.obj * sc.obj          # what the old bug reported
    assert sc.obj != 1.0
    assert not np.allclose(wrong_y, exp.y, rtol=1e-6, atol=1e-9)
