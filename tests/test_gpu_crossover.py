"""Crossover from the engine's PDLP point to an optimal basis.

The reference's ``test_crosses_over_from_the_first_order_point_too``
(``tests/test_crossover.py:106-113``) solves ``random_lp(seed=1)`` with PDLP
at 1e-8, crosses over and demands OPTIMAL with the cold simplex's objective;
here the point comes from the device, and the same is asked on the LPs of the
crossover fixtures up to the 1,200 x 3,600 blending LP, against the
objective of the reference's own cold simplex.
"""

import json
import os
import subprocess
import sys

import numpy as np
import pytest

import crossover_cases as xc
from oracle import verify_oracle as vo
from sovereign_moe_b200 import _lib
from sovereign_moe_b200.crossover import basis_from_point, crossover
from sovereign_moe_b200.mps import read_mps, write_mps
from sovereign_moe_b200.pdlp import PDLPParams, solve_pdlp
from sovereign_moe_b200.problem import Status

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("name", ["random_lp_s1", "random_lp_s3", "badly_scaled_s2", "agree",
                                  "small_known_s0", "blend_mini"])
def test_crosses_over_from_the_device_point(require_gpu, name):
    prob, points, exp = xc.load(name)
    fo = solve_pdlp(prob.copy(), PDLPParams(device="gpu", eps_abs=1e-8, eps_rel=1e-8))
    assert fo.x is not None
    sol = crossover(prob.copy(), fo.x, fo.y)
    assert sol.status == Status.OPTIMAL
    ref = float(exp.cold_objective)
    assert abs(sol.objective - ref) <= 1e-9 * max(1.0, abs(ref))
    assert int((sol.basis_status == _lib.BASIC).sum()) == prob.A.m
    assert sol.info["identified"]["repairs"] == 0


@pytest.mark.parametrize("seed", range(5))
def test_device_point_identifies_the_reference_basis(require_gpu, seed):
    """The engine's point at 1e-8 follows the reference's PDLP trajectory, so
    the basis identified from it is the one the reference identifies from
    its own point."""
    prob, points, exp = xc.load(f"random_lp_s{seed}")
    fo = solve_pdlp(prob.copy(), PDLPParams(device="gpu", eps_abs=1e-8, eps_rel=1e-8))
    assert np.array_equal(basis_from_point(prob, fo.x, fo.y), exp.pdlp_status)


def test_cli_crossover_passes_every_verifier_check(require_gpu, tmp_path):
    """A basic solution closes the gap: with --crossover the verifier's
    certified-gap test (|gap| <= 1e-9 relative) passes too."""
    prob, _, exp = xc.load("small_known_s0")
    model, out = tmp_path / "m.mps", tmp_path / "m.json"
    write_mps(prob, model)
    r = subprocess.run([sys.executable, "-m", "sovereign_moe_b200", "solve", str(model),
                        "--tol", "1e-6", "--crossover", "--out", str(out)],
                       cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    data = json.loads(out.read_text())
    assert data["status"] == "OPTIMAL" and data["method"] == "simplex[primal]"
    ref = float(exp.cold_objective)
    assert abs(data["objective"] - ref) <= 1e-9 * max(1.0, abs(ref))
    v = vo.verify_files(read_mps(model), out, feas_tol=1e-6)
    assert v.ok, v.report()
