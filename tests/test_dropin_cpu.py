"""The drop-in boundary with the caller's own objects (no GPU needed).

``solve_pdlp(prob, params)`` takes the reference's ``Problem`` and
``PDLPParams`` as they are and returns the caller's ``Solution`` / ``Status``
/ ``PDLPInfo`` classes when those come from the reference's package
(``sovopt.core.problem``, ``sovopt.lp.pdlp``).  Here the boundary is checked
without the device: the problem descriptor and the parameter struct built
from the caller's objects, and the result assembly (``_to_solution``) from a
synthetic C result.

The reference itself is used when ``sovopt`` is importable: on the path, or
from the source tree named by the ``SOVOPT_SRC`` environment variable; the
tests that need it skip otherwise.  A stand-in package with the same layout
(``<pkg>.core.problem`` holding ``Problem``, ``Solution``, ``Status``) pins the
class selection either way.
"""

import ctypes
import dataclasses
import enum
import os
import sys
import types

import numpy as np
import pytest

import golden_cases as gc
from sovereign_moe_b200 import _lib
from sovereign_moe_b200 import pdlp as eng_pdlp


def _sovopt():
    """The reference package, or None.  Imported with its JIT cache off and
    no bytecode writes, so nothing is written into its source tree."""
    try:
        import sovopt  # noqa: F401
    except ImportError:
        src = os.environ.get("SOVOPT_SRC")
        if not src or not os.path.isdir(src):
            return None
        os.environ.setdefault("SOVOPT_JIT_CACHE", "0")
        sys.dont_write_bytecode = True
        sys.path.insert(0, src)
        try:
            import sovopt  # noqa: F401
        except ImportError:
            return None
    import sovopt.core.problem as sp
    import sovopt.core.sparse as ss
    import sovopt.lp.pdlp as sl
    return types.SimpleNamespace(problem=sp, sparse=ss, pdlp=sl)


def _fake_result(status, m, n):
    r = _lib.Result()
    r.status, r.iterations, r.restarts, r.rejected_steps = status, 576, 3, 1
    for f in ("primal_res", "dual_res", "gap", "primal_obj", "dual_obj"):
        setattr(r, f, 1e-7)
    r.step_size, r.primal_weight, r.objective, r.scale_obj = 0.5, 2.0, 0.0, 1.0
    r.history_len, r.device_seconds = 1, 0.01
    return r


def _hist():
    return np.array([64.0, 1e-3, 1e-3, 1e-2, 5.0])


def _check_desc(d, prob):
    A = prob.A
    assert (d.m, d.n, d.nnz) == (A.m, A.n, A.nnz)
    for name, arr, ct in (("rp", A.rp, ctypes.c_int64), ("ri", A.ri, ctypes.c_int32),
                          ("rx", A.rx, ctypes.c_double), ("cp", A.cp, ctypes.c_int64),
                          ("ci", A.ci, ctypes.c_int32), ("cx", A.cx, ctypes.c_double),
                          ("c", prob.c, ctypes.c_double), ("row_lb", prob.row_lb, ctypes.c_double),
                          ("row_ub", prob.row_ub, ctypes.c_double),
                          ("col_lb", prob.col_lb, ctypes.c_double),
                          ("col_ub", prob.col_ub, ctypes.c_double)):
        ptr = getattr(d, name)
        got = np.ctypeslib.as_array(ctypes.cast(ptr, ctypes.POINTER(ct)), shape=(len(arr),))
        assert np.array_equal(got, np.asarray(arr)), name
    assert d.sense == (-1 if int(prob.sense) == -1 else 1)
    assert d.obj_offset == float(prob.obj_offset)
    assert d.memory == _lib.PDLP_MEM_HOST


def test_sovopt_problem_and_params_cross_the_boundary():
    so = _sovopt()
    if so is None:
        pytest.skip("sovopt (the reference) is not importable here; set SOVOPT_SRC")
    mine, exp = gc.load("small_known_s0")
    A = so.sparse.SparseMatrix(mine.A.m, mine.A.n, exp.cp, exp.ci, exp.cx)
    prob = so.problem.Problem(A=A, c=exp.c, row_lb=exp.row_lb, row_ub=exp.row_ub,
                              col_lb=exp.col_lb, col_ub=exp.col_ub,
                              obj_offset=float(exp.obj_offset),
                              sense=so.problem.ObjSense(int(exp.sense)))
    params = so.pdlp.PDLPParams(eps_abs=1e-6, eps_rel=1e-6, max_iter=5000, time_limit=30.0,
                                scaling="pdlp")
    d, keep = eng_pdlp.problem_desc(prob)
    _check_desc(d, prob)
    p, _ = eng_pdlp.params_struct(params, prob.A.n)
    for f in ("eps_abs", "eps_rel", "feas_cap", "max_iter", "time_limit", "check_every",
              "stepsize_every", "beta_sufficient", "beta_necessary", "beta_artificial",
              "primal_weight_smoothing"):
        assert getattr(p, f) == getattr(params, f), f
    # the reference's params have no engine-only fields: their defaults apply
    assert p.precision == _lib.PRECISION["fp64"] and p.detect_infeasibility == 0
    # the result comes back in the reference's own classes
    m, n = prob.A.m, prob.A.n
    sol = eng_pdlp._to_solution(prob, params, _fake_result(0, m, n), np.zeros(n), np.zeros(m),
                                np.zeros(n), _hist(), 0.1)
    assert type(sol) is so.problem.Solution
    assert isinstance(sol.status, so.problem.Status) and sol.status == so.problem.Status.OPTIMAL
    assert type(sol.info) is so.pdlp.PDLPInfo
    assert sol.info.history == [(64, 1e-3, 1e-3, 1e-2, 5.0)] and sol.info.device == "gpu"
    assert sol.method == "pdlp[gpu]" and sol.work_units == 576.0
    # an unsolved status drops the objective, as the reference does
    lim = eng_pdlp._to_solution(prob, params, _fake_result(8, m, n), np.zeros(n), np.zeros(m),
                                np.zeros(n), _hist(), 0.1)
    assert lim.status == so.problem.Status.NUMERICAL and np.isnan(lim.objective)


def _standin_package():
    """A caller package laid out like the reference: pkg.core.problem with
    Problem, Solution and Status; pkg.lp.pdlp with PDLPParams and PDLPInfo."""
    prob_mod = types.ModuleType("standin_pkg.core.problem")
    pdlp_mod = types.ModuleType("standin_pkg.lp.pdlp")

    class Status(enum.IntEnum):
        OPTIMAL = 0
        ITERATION_LIMIT = 4
        NUMERICAL = 8

        @property
        def has_solution(self):
            return self in (Status.OPTIMAL, Status.ITERATION_LIMIT)

    @dataclasses.dataclass
    class Solution:
        status: Status
        x: object = None
        objective: float = float("nan")
        y: object = None
        reduced_costs: object = None
        dual_bound: float = float("nan")
        iterations: int = 0
        time: float = 0.0
        work_units: float = 0.0
        method: str = ""
        log: list = dataclasses.field(default_factory=list)

        def drop_objective_if_unsolved(self):
            if not self.status.has_solution:
                self.objective = float("nan")
            return self

    @dataclasses.dataclass
    class Problem:
        A: object
        c: object
        row_lb: object
        row_ub: object
        col_lb: object
        col_ub: object
        obj_offset: float = 0.0
        sense: int = 1

    @dataclasses.dataclass
    class PDLPParams:
        eps_abs: float = 1e-8
        eps_rel: float = 1e-8
        feas_cap: float = 1e-6
        max_iter: int = 200_000
        time_limit: float = 600.0
        check_every: int = 64
        stepsize_every: int = 8
        beta_sufficient: float = 0.2
        beta_necessary: float = 0.8
        beta_artificial: float = 0.36
        primal_weight_smoothing: float = 0.5
        scaling: str = "pdlp"
        device: str = "auto"
        verbose: bool = False
        log_every: int = 2000

    @dataclasses.dataclass
    class PDLPInfo:
        iterations: int = 0
        restarts: int = 0
        rejected_steps: int = 0
        primal_res: float = float("nan")
        dual_res: float = float("nan")
        gap: float = float("nan")
        primal_obj: float = float("nan")
        dual_obj: float = float("nan")
        step_size: float = float("nan")
        primal_weight: float = float("nan")
        device: str = "cpu"
        history: list = dataclasses.field(default_factory=list)

    for cls in (Status, Solution, Problem):
        cls.__module__ = prob_mod.__name__
        setattr(prob_mod, cls.__name__, cls)
    for cls in (PDLPParams, PDLPInfo):
        cls.__module__ = pdlp_mod.__name__
        setattr(pdlp_mod, cls.__name__, cls)
    return prob_mod, pdlp_mod


@pytest.fixture
def standin(monkeypatch):
    prob_mod, pdlp_mod = _standin_package()
    monkeypatch.setitem(sys.modules, prob_mod.__name__, prob_mod)
    monkeypatch.setitem(sys.modules, pdlp_mod.__name__, pdlp_mod)
    return prob_mod, pdlp_mod


def _standin_problem(prob_mod):
    mine, _ = gc.load("toy")
    return prob_mod.Problem(A=mine.A, c=mine.c, row_lb=mine.row_lb, row_ub=mine.row_ub,
                            col_lb=mine.col_lb, col_ub=mine.col_ub,
                            obj_offset=mine.obj_offset, sense=int(mine.sense))


def test_results_come_back_in_the_callers_classes(standin):
    prob_mod, pdlp_mod = standin
    prob = _standin_problem(prob_mod)
    params = pdlp_mod.PDLPParams(eps_abs=1e-6)
    d, keep = eng_pdlp.problem_desc(prob)
    _check_desc(d, prob)
    m, n = prob.A.m, prob.A.n
    sol = eng_pdlp._to_solution(prob, params, _fake_result(0, m, n), np.zeros(n), np.zeros(m),
                                np.zeros(n), _hist(), 0.1)
    assert type(sol) is prob_mod.Solution and sol.status is prob_mod.Status.OPTIMAL
    assert type(sol.info) is pdlp_mod.PDLPInfo and sol.info.device_seconds == 0.01
    lim = eng_pdlp._to_solution(prob, params, _fake_result(8, m, n), np.zeros(n), np.zeros(m),
                                np.zeros(n), _hist(), 0.1)
    assert lim.status is prob_mod.Status.NUMERICAL and np.isnan(lim.objective)


def test_own_objects_get_own_classes():
    from sovereign_moe_b200.problem import Solution, Status
    prob, _ = gc.load("toy")
    params = eng_pdlp.PDLPParams()
    m, n = prob.A.m, prob.A.n
    sol = eng_pdlp._to_solution(prob, params, _fake_result(0, m, n), np.zeros(n), np.zeros(m),
                                np.zeros(n), _hist(), 0.1)
    assert type(sol) is Solution and sol.status is Status.OPTIMAL
    assert type(sol.info) is eng_pdlp.PDLPInfo
