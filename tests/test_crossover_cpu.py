"""Crossover to a basis (host code of the C library; no GPU needed).

Pinned to the reference: ``tests/golden/crossover/`` holds, for the LPs of the
reference's crossover tests and every LP of ``tests/golden/``, the status
vector the reference's ``basis_from_point`` identified from a point, and the
status and objective of its ``crossover`` and of a cold ``solve_simplex``.

The properties the reference's own tests assert (``tests/test_crossover.py``)
are asserted here too: exactly m basic variables, a basis nonsingular by
construction (no repair), a pinned column never basic, the same objective as
a cold simplex, a maximisation handled, and fewer pivots than a cold start
over the set.
"""

import ctypes

import numpy as np
import pytest

import crossover_cases as xc
from oracle import crossover_oracle as xo
from sovereign_moe_b200 import _lib
from sovereign_moe_b200.crossover import basis_from_point, crossover
from sovereign_moe_b200.simplex import SimplexParams, solve_simplex
from sovereign_moe_b200.problem import Status

NAMES = xc.names()
SMALL = [n for n in NAMES if xc.load(n)[0].A.m <= 300]


def _cases():
    for name in NAMES:
        prob, points, exp = xc.load(name)
        for kind in points:
            yield name, kind


CASES = list(_cases())


@pytest.mark.parametrize("name", SMALL)
def test_oracle_identifies_the_reference_basis(name):
    """The dense restatement gives the reference's status vector exactly."""
    prob, points, exp = xc.load(name)
    for kind, (x, y) in points.items():
        work, yy = xc.minimising(prob, y)
        assert np.array_equal(xo.basis_from_point(work, x, yy), exp.__dict__[f"{kind}_status"])


@pytest.mark.parametrize(("name", "kind"), CASES)
def test_identification_matches_the_reference(name, kind):
    """The library's basis_from_point returns the reference's status vector.
    On the blending LP (4,800 variables) two statuses differ: two candidates
    whose pivot entries tie to rounding are taken in the other order, which
    the sparse LU here and the reference's resolve differently."""
    prob, points, exp = xc.load(name)
    x, y = points[kind]
    work, yy = xc.minimising(prob, y)
    got = basis_from_point(work, x, yy)
    want = exp.__dict__[f"{kind}_status"]
    assert int((got == _lib.BASIC).sum()) == prob.A.m
    if name == "blend_mini":
        assert int((got != want).sum()) <= 2
    else:
        assert np.array_equal(got, want)


@pytest.mark.parametrize("name", ["random_lp_s0", "random_lp_s1", "random_lp_s2",
                                  "random_lp_s3", "agree", "small_known_s0"])
def test_identified_basis_is_nonsingular_without_repair(name):
    """The push keeps the basis nonsingular at every step: the library reports
    no repair, and the dense basis matrix of the result is well inside
    double precision."""
    prob, points, _ = xc.load(name)
    x, y = points["pdlp"]
    desc, keep = _desc(prob)
    st = np.zeros(prob.A.n + prob.A.m, dtype=np.uint8)
    info = _lib.CrossoverInfo()
    lib = _lib.load()
    _lib.check(lib.pdlp_basis_from_point(ctypes.byref(desc), np.ascontiguousarray(x).ctypes.data,
                                         np.ascontiguousarray(y).ctypes.data, 1e-12, 1e-7,
                                         st.ctypes.data, ctypes.byref(info)))
    assert info.repairs == 0 and info.placed + info.rejected <= info.candidates
    M = xo._dense_M(prob)
    assert np.linalg.cond(M[:, st == _lib.BASIC]) < 1e12


def test_a_fixed_variable_is_never_made_basic():
    prob, points, _ = xc.load("pinned")
    x, y = points["ipm"]
    st = basis_from_point(prob, x, y)
    assert prob.col_lb[1] == prob.col_ub[1] and st[1] == _lib.FIXED


@pytest.mark.parametrize(("name", "kind"), CASES)
def test_crossover_agrees_with_the_reference(name, kind):
    """Same status as the reference's cold simplex and the same objective
    (rel 1e-9), at a basis that is primal and dual feasible when rebuilt
    densely from its status vector."""
    prob, points, exp = xc.load(name)
    x, y = points[kind]
    sol = crossover(prob.copy(), x, y)
    assert int(sol.status) == int(exp.cold_status)
    assert sol.info["crossover"] is True
    if int(exp.cold_status) != 0:
        return
    ref = float(exp.cold_objective)
    assert abs(sol.objective - ref) <= 1e-9 * max(1.0, abs(ref))
    assert int((sol.basis_status == _lib.BASIC).sum()) == prob.A.m
    if prob.A.m <= 300:
        work, _ = xc.minimising(prob, y)
        bx, _, _, p_inf, d_inf = xo.kkt_of_basis(prob, sol.basis_status, minimise_c=work.c)
        scale = max(1.0, np.abs(prob.c).max())
        assert p_inf <= 1e-6 and d_inf <= 1e-6 * scale
        np.testing.assert_allclose(sol.x, np.clip(bx, prob.col_lb, prob.col_ub),
                                   rtol=1e-7, atol=1e-7)


def test_a_maximisation_crosses_over_to_its_optimum():
    prob, points, _ = xc.load("toy_max")
    x, y = points["ipm"]
    sol = crossover(prob, x, y)
    assert sol.status == Status.OPTIMAL and abs(sol.objective - 11.0) < 1e-9
    np.testing.assert_allclose(sol.x, [3.0, 1.0], atol=1e-9)


@pytest.mark.parametrize("name", NAMES)
def test_cold_simplex_agrees_with_the_reference(name):
    prob, _, exp = xc.load(name)
    sol = solve_simplex(prob.copy(), SimplexParams())
    assert int(sol.status) == int(exp.cold_status)
    if int(exp.cold_status) == 0:
        ref = float(exp.cold_objective)
        assert abs(sol.objective - ref) <= 1e-9 * max(1.0, abs(ref))


def test_crossover_saves_pivots_against_a_cold_start():
    """In aggregate, as the reference asserts it: crossing over from the PDLP
    point must cost fewer pivots than solving from the slack basis."""
    cold = xover = 0
    for name in ("agree", "small_known_s0", "small_known_s1", "small_known_iterlimit",
                 "blend_mini"):
        prob, points, _ = xc.load(name)
        x, y = points["pdlp"]
        c = solve_simplex(prob.copy())
        s = crossover(prob.copy(), x, y)
        assert c.status == Status.OPTIMAL and s.status == Status.OPTIMAL
        cold += c.iterations
        xover += s.iterations
    assert xover < cold, (xover, cold)


def test_warm_start_from_an_optimal_basis_takes_no_pivots():
    prob, points, _ = xc.load("small_known_s0")
    first = solve_simplex(prob.copy())
    again = solve_simplex(prob.copy(), warm_basis=first.basis_status)
    assert again.status == Status.OPTIMAL and again.iterations == 0
    assert again.objective == pytest.approx(first.objective, rel=1e-12)


def _desc(prob):
    from sovereign_moe_b200.pdlp import problem_desc
    return problem_desc(prob)


def test_argument_errors_are_reported():
    lib = _lib.load()
    prob, points, _ = xc.load("toy")
    desc, keep = _desc(prob)
    n, m = prob.A.n, prob.A.m
    st = np.zeros(n + m, dtype=np.uint8)
    x = np.zeros(n)
    assert lib.pdlp_basis_from_point(None, x.ctypes.data, None, 1e-12, 1e-7, st.ctypes.data,
                                     None) == _lib.PDLP_ERR_ARG
    bad = np.full(n, np.nan)
    assert lib.pdlp_basis_from_point(ctypes.byref(desc), bad.ctypes.data, None, 1e-12, 1e-7,
                                     st.ctypes.data, None) == _lib.PDLP_ERR_NUMERICAL
    desc.memory = _lib.PDLP_MEM_DEVICE
    assert lib.pdlp_basis_from_point(ctypes.byref(desc), x.ctypes.data, None, 1e-12, 1e-7,
                                     st.ctypes.data, None) == _lib.PDLP_ERR_ARG
    desc.memory = _lib.PDLP_MEM_HOST
    y, d = np.zeros(m), np.zeros(n)
    warm = np.full(n + m, 9, dtype=np.uint8)
    assert lib.pdlp_simplex_solve(ctypes.byref(desc), None, warm.ctypes.data, x.ctypes.data,
                                  y.ctypes.data, d.ctypes.data, st.ctypes.data,
                                  None) == _lib.PDLP_ERR_ARG
    p = _lib.SimplexParamsC()
    assert lib.pdlp_simplex_default_params(ctypes.byref(p)) == 0
    assert (p.feas_tol, p.opt_tol, p.pivot_tol, p.max_iter, p.time_limit, p.refactor_freq) == \
        (1e-7, 1e-7, 1e-7, 1_000_000, 300.0, 150)
    p.feas_tol = 0.0
    assert lib.pdlp_simplex_solve(ctypes.byref(desc), ctypes.byref(p), None, x.ctypes.data,
                                  y.ctypes.data, d.ctypes.data, st.ctypes.data,
                                  None) == _lib.PDLP_ERR_ARG
