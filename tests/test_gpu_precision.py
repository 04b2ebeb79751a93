"""Float32-SpMV iteration and float64 iterative refinement.

* ``precision="fp32"``: the iteration's sparse products run in float32
  (values, gathered directions, row sums); iterates, restarts and every
  termination quantity stay float64, and termination is the reference's test
  on the unscaled problem.  The results must meet the same bars as the
  float64 engine: status, objective within 1e-6 relative of the reference's
  and of the known optimum, verifier acceptance at 1e-6.
* ``solve_refined``: float32 inner solves at 1e-4 plus float64 refinement to
  rel KKT 1e-8; the objective must match the known optimum to 1e-8 and the
  point must pass the verifier at 1e-8.
"""

import numpy as np
import pytest

import golden_cases as gc
from oracle import verify_oracle as vo
from sovereign_moe_b200 import workloads
from sovereign_moe_b200.pdlp import PDLPParams, solve_pdlp
from sovereign_moe_b200.problem import Status

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["small_known_s0", "small_known_s1", "agree", "toy",
                                  "testprob", "dual_regression"])
def test_fp32_spmv_matches_reference(require_gpu, name):
    prob, exp = gc.load(name)
    s = solve_pdlp(prob, PDLPParams(device="gpu", precision="fp32", **gc.PARAMS[name]))
    assert s.status == Status.OPTIMAL
    ref = float(exp.objective)
    assert abs(s.objective - ref) / max(1.0, abs(ref)) < 1e-6
    if np.isfinite(exp.known):
        assert abs(s.objective - float(exp.known)) / max(1.0, abs(float(exp.known))) < 1e-6
    v = vo.verify(prob, s.x, s.objective, feas_tol=1e-6)
    assert v.ok, v.report()


@pytest.mark.parametrize("seed", [0, 3])
def test_refinement_reaches_1e8(require_gpu, seed):
    from sovereign_moe_b200.refine import solve_refined
    k = workloads.single_small(seed=seed)
    s = solve_refined(k.problem, PDLPParams(device="gpu"), target=1e-8)
    assert s.status == Status.OPTIMAL, s.log
    assert abs(s.objective - k.f_star) / max(1.0, abs(k.f_star)) < 1e-8
    v = vo.verify(k.problem, s.x, s.objective, feas_tol=1e-8)
    assert v.ok, v.report()
    assert len(s.log) <= 6


def test_refinement_with_inequality_rows(require_gpu):
    """Slack columns carry the row ranges; max sense flips back."""
    from sovereign_moe_b200.refine import solve_refined
    prob, _ = gc.load("toy")            # max 3x + 2y, <= rows, optimum 11
    s = solve_refined(prob, PDLPParams(device="gpu"), target=1e-9)
    assert s.status == Status.OPTIMAL
    assert abs(s.objective - 11.0) < 1e-8
    assert np.allclose(s.x, [3.0, 1.0], atol=1e-7)
