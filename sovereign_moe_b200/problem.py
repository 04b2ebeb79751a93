"""Model and result types of the PDLP path.

These keep the field names, enum values and conventions of the reference's
``sovopt`` types, so a caller of ``sovopt.lp.pdlp.solve_pdlp`` can hand the
same objects to :func:`sovereign_moe_b200.solve_pdlp` (and the reference's own
``Problem`` objects are accepted as they are -- only attributes are read):

* ``Problem``        -- row-bounds form ``rl <= Ax <= ru, l <= x <= u``
  (``src/sovopt/core/problem.py:81-275``);
* ``Solution``       -- ``src/sovopt/core/problem.py:278-343``, including
  ``drop_objective_if_unsolved``;
* ``Status``, ``ObjSense``, ``VarKind`` -- same integers (``problem.py:45-78``);
* ``SparseMatrix``   -- one matrix held in CSC and CSR at once, int64
  pointers, int32 indices, float64 values (``src/sovopt/core/sparse.py:263-298``);
* ``INF = 1e30``     -- the infinite-bound sentinel (``core/tolerances.py:16``).

Host-side products here are plain NumPy: they serve model construction and
reporting, not the solve, which runs on the GPU.
"""

from __future__ import annotations

from dataclasses import dataclass, field
from enum import IntEnum

import numpy as np

__all__ = ["INF", "VarKind", "ObjSense", "Status", "SparseMatrix", "Problem",
           "Solution"]

INF = 1.0e30
IDX = np.int32
VAL = np.float64


class VarKind(IntEnum):
    CONTINUOUS = 0
    INTEGER = 1
    BINARY = 2
    SEMI_CONTINUOUS = 3
    SEMI_INTEGER = 4


class ObjSense(IntEnum):
    MINIMISE = 1
    MAXIMISE = -1


class Status(IntEnum):
    OPTIMAL = 0
    INFEASIBLE = 1
    UNBOUNDED = 2
    INFEASIBLE_OR_UNBOUNDED = 3
    ITERATION_LIMIT = 4
    TIME_LIMIT = 5
    NODE_LIMIT = 6
    GAP_LIMIT = 7
    NUMERICAL = 8
    INTERRUPTED = 9
    NOT_SOLVED = 10

    @property
    def is_solved(self) -> bool:
        return self in (Status.OPTIMAL,)

    @property
    def has_solution(self) -> bool:
        return self in (Status.OPTIMAL, Status.ITERATION_LIMIT, Status.TIME_LIMIT,
                        Status.NODE_LIMIT, Status.GAP_LIMIT)


def _transpose(indptr, indices, values, n_other):
    """Transpose compressed storage by a stable sort on the target index, so
    every target slice lists its entries in increasing source-slice order (the
    order a counting sort gives, ``src/sovopt/core/sparse.py:148-172``)."""
    n = indptr.shape[0] - 1
    nnz = indices.shape[0]
    src = np.repeat(np.arange(n, dtype=IDX), np.diff(indptr))
    order = np.argsort(indices, kind="stable")
    t_indptr = np.zeros(n_other + 1, dtype=np.int64)
    if nnz:
        np.cumsum(np.bincount(indices, minlength=n_other), out=t_indptr[1:])
    return t_indptr, np.ascontiguousarray(src[order]), np.ascontiguousarray(values[order])


def coo_to_csc(rows, cols, vals, m: int, n: int, sum_duplicates: bool = True):
    """CSC arrays from triplets: sorted by (column, row), exact duplicates
    summed, explicit zeros dropped (``src/sovopt/core/sparse.py:198-236``)."""
    rows = np.asarray(rows, dtype=IDX)
    cols = np.asarray(cols, dtype=IDX)
    vals = np.asarray(vals, dtype=VAL)
    if rows.shape != cols.shape or rows.shape != vals.shape:
        raise ValueError("triplet arrays must have equal length")
    order = np.lexsort((rows, cols))
    rows, cols, vals = rows[order], cols[order], vals[order]
    if sum_duplicates and rows.size:
        keyed = cols.astype(np.int64) * np.int64(m) + rows.astype(np.int64)
        first = np.empty(keyed.shape[0], dtype=bool)
        first[0] = True
        np.not_equal(keyed[1:], keyed[:-1], out=first[1:])
        if not first.all():
            group = np.cumsum(first) - 1
            vals = np.bincount(group, weights=vals)
            rows, cols = rows[first], cols[first]
    keep = vals != 0.0
    if not keep.all():
        rows, cols, vals = rows[keep], cols[keep], vals[keep]
    indptr = np.zeros(n + 1, dtype=np.int64)
    if cols.size:
        np.add.at(indptr, cols.astype(np.int64) + 1, 1)
    np.cumsum(indptr, out=indptr)
    return indptr, np.ascontiguousarray(rows), np.ascontiguousarray(vals)


class SparseMatrix:
    """An ``m x n`` sparse matrix held in CSC and CSR at once."""

    __slots__ = ("m", "n", "cp", "ci", "cx", "rp", "ri", "rx")

    def __init__(self, m: int, n: int, cp, ci, cx, rp=None, ri=None, rx=None):
        self.m = int(m)
        self.n = int(n)
        self.cp = np.ascontiguousarray(cp, dtype=np.int64)
        self.ci = np.ascontiguousarray(ci, dtype=IDX)
        self.cx = np.ascontiguousarray(cx, dtype=VAL)
        if rp is None:
            rp, ri, rx = _transpose(self.cp, self.ci, self.cx, self.m)
        self.rp = np.ascontiguousarray(rp, dtype=np.int64)
        self.ri = np.ascontiguousarray(ri, dtype=IDX)
        self.rx = np.ascontiguousarray(rx, dtype=VAL)

    @classmethod
    def from_triplets(cls, rows, cols, vals, m: int, n: int) -> "SparseMatrix":
        cp, ci, cx = coo_to_csc(rows, cols, vals, m, n)
        return cls(m, n, cp, ci, cx)

    @classmethod
    def from_dense(cls, A) -> "SparseMatrix":
        A = np.asarray(A, dtype=VAL)
        rows, cols = np.nonzero(A)
        return cls.from_triplets(rows, cols, A[rows, cols], A.shape[0], A.shape[1])

    @property
    def shape(self):
        return (self.m, self.n)

    @property
    def nnz(self) -> int:
        return int(self.ci.shape[0])

    def matvec(self, x):
        """``A @ x`` (host, NumPy)."""
        x = np.asarray(x, dtype=VAL)
        rows = np.repeat(np.arange(self.m), np.diff(self.rp))
        return np.bincount(rows, weights=self.rx * x[self.ri], minlength=self.m)

    def rmatvec(self, y):
        """``Aᵀ @ y`` (host, NumPy)."""
        y = np.asarray(y, dtype=VAL)
        cols = np.repeat(np.arange(self.n), np.diff(self.cp))
        return np.bincount(cols, weights=self.cx * y[self.ci], minlength=self.n)

    def copy(self) -> "SparseMatrix":
        return SparseMatrix(self.m, self.n, self.cp.copy(), self.ci.copy(), self.cx.copy(),
                            self.rp.copy(), self.ri.copy(), self.rx.copy())

    def to_dense(self):
        A = np.zeros((self.m, self.n), dtype=VAL)
        cols = np.repeat(np.arange(self.n), np.diff(self.cp))
        A[self.ci, cols] = self.cx
        return A

    def __repr__(self):
        return f"SparseMatrix({self.m}x{self.n}, nnz={self.nnz})"


@dataclass
class Problem:
    """An LP in row-bounds form (``src/sovopt/core/problem.py:81-128``)."""

    A: SparseMatrix
    c: np.ndarray
    row_lb: np.ndarray
    row_ub: np.ndarray
    col_lb: np.ndarray
    col_ub: np.ndarray
    kind: np.ndarray = None
    Q: object = None
    obj_offset: float = 0.0
    sense: ObjSense = ObjSense.MINIMISE
    name: str = "model"
    col_names: list | None = None
    row_names: list | None = None
    meta: dict = field(default_factory=dict)

    def __post_init__(self):
        self.c = np.ascontiguousarray(self.c, dtype=VAL)
        self.row_lb = np.ascontiguousarray(self.row_lb, dtype=VAL)
        self.row_ub = np.ascontiguousarray(self.row_ub, dtype=VAL)
        self.col_lb = np.ascontiguousarray(self.col_lb, dtype=VAL)
        self.col_ub = np.ascontiguousarray(self.col_ub, dtype=VAL)
        if self.kind is None:
            self.kind = np.zeros(self.n, dtype=np.uint8)
        else:
            self.kind = np.ascontiguousarray(self.kind, dtype=np.uint8)
        m, n = self.A.shape
        for arr, size, what in ((self.c, n, "c"), (self.col_lb, n, "col_lb"),
                                (self.col_ub, n, "col_ub"), (self.kind, n, "kind"),
                                (self.row_lb, m, "row_lb"), (self.row_ub, m, "row_ub")):
            if arr.shape[0] != size:
                raise ValueError(f"{what} has length {arr.shape[0]}, expected {size}")

    @property
    def m(self) -> int:
        return self.A.m

    @property
    def n(self) -> int:
        return self.A.n

    @property
    def nnz(self) -> int:
        return self.A.nnz

    def objective(self, x) -> float:
        return float(self.c @ np.asarray(x, dtype=VAL)) + self.obj_offset

    def violation(self, x):
        """``(max row violation, max bound violation, 0.0)`` (problem.py:190-206)."""
        x = np.asarray(x, dtype=VAL)
        act = self.A.matvec(x)
        row_v = max(float(np.maximum(self.row_lb - act, 0.0).max(initial=0.0)),
                    float(np.maximum(act - self.row_ub, 0.0).max(initial=0.0)))
        col_v = max(float(np.maximum(self.col_lb - x, 0.0).max(initial=0.0)),
                    float(np.maximum(x - self.col_ub, 0.0).max(initial=0.0)))
        return row_v, col_v, 0.0

    def copy(self) -> "Problem":
        return Problem(A=self.A.copy(), c=self.c.copy(), row_lb=self.row_lb.copy(),
                       row_ub=self.row_ub.copy(), col_lb=self.col_lb.copy(),
                       col_ub=self.col_ub.copy(), kind=self.kind.copy(), Q=self.Q,
                       obj_offset=self.obj_offset, sense=self.sense, name=self.name,
                       meta=dict(self.meta))


@dataclass
class Solution:
    """Result of a solve (``src/sovopt/core/problem.py:278-343``)."""

    status: Status
    x: np.ndarray | None = None
    objective: float = float("nan")
    y: np.ndarray | None = None
    reduced_costs: np.ndarray | None = None
    basis_status: np.ndarray | None = None
    dual_bound: float = float("nan")
    nodes: int = 0
    gap_rel: float = float("nan")
    iterations: int = 0
    time: float = 0.0
    work_units: float = 0.0
    method: str = ""
    log: list = field(default_factory=list)
    sensitivity: object = None
    farkas: np.ndarray | None = None
    info: object = None

    def drop_objective_if_unsolved(self) -> "Solution":
        """NaN objective and bound unless the status carries a point."""
        if not Status(self.status).has_solution:
            self.objective = float("nan")
            self.dual_bound = float("nan")
        return self

    @property
    def gap(self) -> float:
        if not np.isfinite(self.objective) or not np.isfinite(self.dual_bound):
            return float("inf")
        return abs(self.objective - self.dual_bound) / max(1.0, abs(self.objective))

    def __repr__(self):
        obj = f"{self.objective:.10g}" if np.isfinite(self.objective) else "-"
        return (f"Solution({Status(self.status).name}, obj={obj}, "
                f"iters={self.iterations}, {self.time:.3f}s)")
