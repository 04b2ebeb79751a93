"""CPU restatement of the reference PDLP path -- TEST INFRASTRUCTURE ONLY.

Restarted averaged PDHG exactly as ``src/sovopt/lp/pdlp.py`` runs it with
``device="cpu"``, and the ``method="pdlp"`` preconditioner of
``src/sovopt/numerics/scaling.py``.  The array expressions are the same NumPy
calls the reference makes on its CPU backend, and the sparse kernels
(``oracle/sparse_ref.c``) accumulate in the reference's order, so a solve here
follows the reference's iterate sequence bit for bit (pinned by
``tests/test_oracle_golden.py`` against outputs of the reference itself).

The problem object is duck-typed: anything with ``A`` (``m, n, cp, ci, cx,
rp, ri, rx``), ``c, row_lb, row_ub, col_lb, col_ub, obj_offset, sense`` works
-- the reference's ``Problem``, the product's, or a fixture record.
"""

from __future__ import annotations

import ctypes
import os
import time
from dataclasses import dataclass, field
from types import SimpleNamespace

import numpy as np

INF = 1.0e30                       # src/sovopt/core/tolerances.py:16

# Status codes, same integers as src/sovopt/core/problem.py:58-69
OPTIMAL, ITERATION_LIMIT, TIME_LIMIT, NUMERICAL = 0, 4, 5, 8
STATUS_NAMES = {0: "OPTIMAL", 1: "INFEASIBLE", 2: "UNBOUNDED",
                3: "INFEASIBLE_OR_UNBOUNDED", 4: "ITERATION_LIMIT",
                5: "TIME_LIMIT", 6: "NODE_LIMIT", 7: "GAP_LIMIT",
                8: "NUMERICAL", 9: "INTERRUPTED", 10: "NOT_SOLVED"}
_HAS_SOLUTION = {0, 4, 5, 6, 7}    # problem.py:75-78
MAXIMISE = -1

# --------------------------------------------------------------------------- #
# C kernels                                                                    #
# --------------------------------------------------------------------------- #

_LIB = None
_HERE = os.path.dirname(os.path.abspath(__file__))


def lib():
    """The oracle's C kernels (``oracle/liboracle_sparse.so``), built on demand."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = os.path.join(_HERE, "liboracle_sparse.so")
    if not os.path.exists(path):
        import subprocess
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    L = ctypes.CDLL(path)
    i64, p = ctypes.c_int64, ctypes.c_void_p
    L.csr_spmv.argtypes = [i64, p, p, p, p, p]
    L.abs_max_by_slice.argtypes = [i64, p, p, p]
    L.scale_csc.argtypes = [i64, p, p, p, p, p]
    L.scale_csr.argtypes = [i64, p, p, p, p, p]
    L.transpose.argtypes = [i64, p, p, p, i64, p, p, p]
    L.transpose.restype = ctypes.c_int
    L.residual_csr.argtypes = [i64, p, p, p, p, p, p]
    L.csr_spmm.argtypes = [i64, i64, p, p, p, p, p]
    L.oracle_num_threads.restype = ctypes.c_int
    L.oracle_set_threads.argtypes = [ctypes.c_int]
    _LIB = L
    return L


def _ptr(a):
    return a.ctypes.data


def num_threads() -> int:
    return int(lib().oracle_num_threads())


def set_threads(n: int) -> None:
    lib().oracle_set_threads(int(n))


def spmv(indptr, indices, values, x, out=None):
    """``out[i] = Σ_p values[p]·x[indices[p]]`` over slice ``i`` (sparse.py:50-58)."""
    ns = indptr.shape[0] - 1
    x = np.ascontiguousarray(x, dtype=np.float64)
    if out is None:
        out = np.empty(ns, dtype=np.float64)
    lib().csr_spmv(ns, _ptr(indptr), _ptr(indices), _ptr(values), _ptr(x), _ptr(out))
    return out


def spmm(indptr, indices, values, X, out=None):
    """``out = A X`` with ``X`` dense ``(n, k)`` row-major (sparse.py:72-84)."""
    X = np.ascontiguousarray(X, dtype=np.float64)
    ns, k = indptr.shape[0] - 1, X.shape[1]
    if out is None:
        out = np.empty((ns, k), dtype=np.float64)
    lib().csr_spmm(ns, k, _ptr(indptr), _ptr(indices), _ptr(values), _ptr(X), _ptr(out))
    return out


def abs_max_by_slice(indptr, values):
    ns = indptr.shape[0] - 1
    out = np.empty(ns, dtype=np.float64)
    lib().abs_max_by_slice(ns, _ptr(indptr), _ptr(values), _ptr(out))
    return out


def transpose(indptr, indices, values, n_other):
    """Counting-sort transpose, CSC <-> CSR (sparse.py:148-172, 239-255)."""
    n = indptr.shape[0] - 1
    nnz = indices.shape[0]
    t_indptr = np.zeros(n_other + 1, dtype=np.int64)
    t_indices = np.empty(nnz, dtype=np.int32)
    t_values = np.empty(nnz, dtype=np.float64)
    rc = lib().transpose(n, _ptr(indptr), _ptr(indices), _ptr(values), n_other,
                         _ptr(t_indptr), _ptr(t_indices), _ptr(t_values))
    if rc != 0:
        raise MemoryError("transpose: allocation failed")
    return t_indptr, t_indices, t_values


def compensated_residual(rp, ri, rx, x, b):
    """``b - A x`` to about double-double accuracy (refine.py:49-87, 113-120)."""
    m = rp.shape[0] - 1
    out = np.empty(m, dtype=np.float64)
    x = np.ascontiguousarray(x, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    lib().residual_csr(m, _ptr(rp), _ptr(ri), _ptr(rx), _ptr(x), _ptr(b), _ptr(out))
    return out


# --------------------------------------------------------------------------- #
# sparse matrix in both storage orders                                         #
# --------------------------------------------------------------------------- #


class Mat:
    """CSC + CSR arrays of one matrix, as ``SparseMatrix`` holds them
    (sparse.py:263-298): int64 pointers, int32 indices, float64 values."""

    def __init__(self, m, n, cp, ci, cx, rp=None, ri=None, rx=None):
        self.m, self.n = int(m), int(n)
        self.cp = np.ascontiguousarray(cp, dtype=np.int64)
        self.ci = np.ascontiguousarray(ci, dtype=np.int32)
        self.cx = np.ascontiguousarray(cx, dtype=np.float64)
        if rp is None:
            rp, ri, rx = transpose(self.cp, self.ci, self.cx, self.m)
        self.rp = np.ascontiguousarray(rp, dtype=np.int64)
        self.ri = np.ascontiguousarray(ri, dtype=np.int32)
        self.rx = np.ascontiguousarray(rx, dtype=np.float64)

    @classmethod
    def of(cls, A):
        return cls(A.m, A.n, A.cp, A.ci, A.cx, A.rp, A.ri, A.rx)

    @property
    def nnz(self):
        return int(self.ci.shape[0])

    def copy(self):
        return Mat(self.m, self.n, self.cp.copy(), self.ci.copy(), self.cx.copy(),
                   self.rp.copy(), self.ri.copy(), self.rx.copy())

    def matvec(self, x):
        return spmv(self.rp, self.ri, self.rx, x)

    def rmatvec(self, y):
        return spmv(self.cp, self.ci, self.cx, y)

    def row_absmax(self):
        return abs_max_by_slice(self.rp, self.rx)

    def col_absmax(self):
        return abs_max_by_slice(self.cp, self.cx)

    def scale(self, r, c):
        """In place ``A <- diag(r) A diag(c)`` on both forms (sparse.py:472-485)."""
        r = np.ascontiguousarray(r, dtype=np.float64)
        c = np.ascontiguousarray(c, dtype=np.float64)
        L = lib()
        L.scale_csc(self.n, _ptr(self.cp), _ptr(self.ci), _ptr(self.cx), _ptr(r), _ptr(c))
        L.scale_csr(self.m, _ptr(self.rp), _ptr(self.ri), _ptr(self.rx), _ptr(r), _ptr(c))


# --------------------------------------------------------------------------- #
# scaling  (src/sovopt/numerics/scaling.py)                                    #
# --------------------------------------------------------------------------- #


@dataclass
class Scaling:
    """scaling.py:65-112."""
    row: np.ndarray
    col: np.ndarray
    obj: float = 1.0
    rhs: float = 1.0
    unit: float = 1.0
    method: str = "none"

    def unscale_primal(self, x_scaled):
        return np.asarray(x_scaled, dtype=np.float64) * self.col

    def unscale_dual(self, y_scaled):
        # division by the objective scale, scaling.py:94-108
        return np.asarray(y_scaled, dtype=np.float64) * self.row / (self.obj / self.rhs)


def pow2_round(s):
    """scaling.py:119-131."""
    s = np.asarray(s, dtype=np.float64)
    out = np.ones_like(s)
    good = np.isfinite(s) & (s > 0.0)
    if good.any():
        out[good] = np.exp2(np.rint(np.log2(s[good])))
    return out


def ruiz(A: Mat, iters=20, tol=1e-2):
    """∞-norm equilibration, scaling.py:149-170."""
    r = np.ones(A.m)
    c = np.ones(A.n)
    W = A.copy()
    for _ in range(iters):
        rmax = W.row_absmax()
        cmax = W.col_absmax()
        rmax[rmax <= 0.0] = 1.0
        cmax[cmax <= 0.0] = 1.0
        dev = max(float(np.abs(1.0 - rmax).max(initial=0.0)),
                  float(np.abs(1.0 - cmax).max(initial=0.0)))
        dr = 1.0 / np.sqrt(rmax)
        dc = 1.0 / np.sqrt(cmax)
        W.scale(dr, dc)
        r *= dr
        c *= dc
        if dev < tol:
            break
    return r, c


def pock_chambolle(A: Mat):
    """Pock-Chambolle with alpha = 1, scaling.py:274-295.

    The reference builds a matrix of |a_ij| from the CSC arrays and sums it
    with its CSR kernel (rows, column order) and its CSC kernel (columns, row
    order); the same two passes run here."""
    absx = np.abs(A.cx)
    rp, ri, rabs = transpose(A.cp, A.ci, absx, A.m)
    rsum = spmv(rp, ri, rabs, np.ones(A.n))
    csum = spmv(A.cp, A.ci, absx, np.ones(A.m))
    rsum[rsum <= 0.0] = 1.0
    csum[csum <= 0.0] = 1.0
    return 1.0 / np.sqrt(rsum), 1.0 / np.sqrt(csum)


def pdlp_scaling(A: Mat, ruiz_iters=10):
    """Ruiz then Pock-Chambolle, scaling.py:298-309."""
    r, c = ruiz(A, iters=ruiz_iters)
    W = A.copy()
    W.scale(r, c)
    r2, c2 = pock_chambolle(W)
    return r * r2, c * c2


_METHODS = {"pdlp": pdlp_scaling, "ruiz": ruiz, "pock_chambolle": pock_chambolle}


def scale_problem(prob, method="pdlp"):
    """``scale_problem(prob, method)`` for an LP, scaling.py:374-478 with
    ``compute_scaling`` (321-371): pow2 factors, columns of a non-continuous
    ``kind`` pinned to 1 (scaling.py:353-355, 401), objective scale from the
    nonzero costs, infinite bounds kept infinite.

    Returns ``(S, sc)`` where ``S`` is a namespace with the scaled ``A``
    (a :class:`Mat`), ``c, row_lb, row_ub, col_lb, col_ub, obj_offset``."""
    A0 = Mat.of(prob.A)
    if method in ("none", None):
        r, c = np.ones(A0.m), np.ones(A0.n)
        meth = "none"
    else:
        if method not in _METHODS:
            raise ValueError(f"oracle supports scaling {sorted(_METHODS)} or 'none'")
        r, c = _METHODS[method](A0)
        r, c = pow2_round(r), pow2_round(c)
        kind = getattr(prob, "kind", None)
        if kind is not None and np.any(np.asarray(kind) != 0):
            c = c.copy()
            c[np.asarray(kind) != 0] = 1.0
        meth = method
    sc = Scaling(r, c, method=meth)
    A = A0.copy()
    A.scale(sc.row, sc.col)
    cc = np.asarray(prob.c, dtype=np.float64) * sc.col
    nz = np.abs(cc[cc != 0.0])
    obj_scale = 1.0
    if nz.size:
        g = float(np.exp2(np.rint(np.log2(np.sqrt(nz.max() * nz.min())))))
        if g > 0 and np.isfinite(g):
            obj_scale = 1.0 / g
    cc = cc * obj_scale
    sc.obj = obj_scale

    def row_bound(b, s):
        out = b * s
        out[b <= -INF] = -INF
        out[b >= INF] = INF
        return out

    def col_bound(b, s):
        out = b / s
        out[b <= -INF] = -INF
        out[b >= INF] = INF
        return out

    S = SimpleNamespace(
        A=A, c=cc,
        row_lb=row_bound(np.asarray(prob.row_lb, dtype=np.float64), sc.row),
        row_ub=row_bound(np.asarray(prob.row_ub, dtype=np.float64), sc.row),
        col_lb=col_bound(np.asarray(prob.col_lb, dtype=np.float64), sc.col),
        col_ub=col_bound(np.asarray(prob.col_ub, dtype=np.float64), sc.col),
        obj_offset=float(prob.obj_offset) * obj_scale,
        m=A.m, n=A.n)
    return S, sc


# --------------------------------------------------------------------------- #
# PDLP  (src/sovopt/lp/pdlp.py)                                                #
# --------------------------------------------------------------------------- #


@dataclass
class Params:
    """pdlp.py:79-116 (same field names and defaults)."""
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
    device: str = "cpu"
    verbose: bool = False
    log_every: int = 2000


@dataclass
class Info:
    """pdlp.py:119-132."""
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
    history: list = field(default_factory=list)


def _param(params, name):
    if params is None:
        return getattr(Params, name)
    if isinstance(params, dict):
        return params.get(name, getattr(Params, name))
    return getattr(params, name, getattr(Params, name))


def estimate_norm(A: Mat, iters=20):
    """Power iteration for ‖A‖₂ from ``default_rng(0)`` (pdlp.py:140-159)."""
    rng = np.random.default_rng(0)
    v = rng.standard_normal(A.n)
    nv = float(np.linalg.norm(v))
    if nv == 0.0:
        return 1.0
    v /= nv
    est = 1.0
    for _ in range(iters):
        av = A.matvec(v)
        atv = A.rmatvec(av)
        nrm = float(np.linalg.norm(atv))
        if nrm <= 0.0:
            return 1.0
        v = atv / nrm
        est = np.sqrt(nrm)
    return float(max(est, 1e-12))


class KKT:
    """Scaled KKT residuals of a primal-dual pair (pdlp.py:162-230)."""

    def __init__(self, S):
        self.S = S
        self.ru_fin = S.row_ub < INF
        self.rl_fin = S.row_lb > -INF
        self.lo_fin = S.col_lb > -INF
        self.hi_fin = S.col_ub < INF

    def __call__(self, x, y, ax=None, aty=None):
        S = self.S
        if ax is None:
            ax = S.A.matvec(x)
        if aty is None:
            aty = S.A.rmatvec(y)
        pv = np.maximum(S.row_lb - ax, 0.0) + np.maximum(ax - S.row_ub, 0.0)
        primal_res = float(np.abs(pv).max()) if S.m else 0.0
        d = S.c + aty
        dpos = np.maximum(d, 0.0)
        dneg = np.maximum(-d, 0.0)
        dres = np.where(self.lo_fin, 0.0, dpos) + np.where(self.hi_fin, 0.0, dneg)
        dual_res = float(np.abs(dres).max()) if S.n else 0.0
        primal_obj = float(np.dot(S.c, x)) + S.obj_offset
        supp = (np.where(y > 0.0, np.where(self.ru_fin, S.row_ub, 0.0),
                         np.where(self.rl_fin, S.row_lb, 0.0)) * y)
        bnd = (np.where(d > 0.0, np.where(self.lo_fin, S.col_lb, 0.0),
                        np.where(self.hi_fin, S.col_ub, 0.0)) * d)
        dual_obj = float(-np.sum(supp) + np.sum(bnd)) + S.obj_offset
        gap = abs(primal_obj - dual_obj)
        return primal_res, dual_res, gap, primal_obj, dual_obj

    def merit(self, x, y, omega, ax=None, aty=None):
        p, dres, g, _, _ = self(x, y, ax, aty)
        return float(np.sqrt((omega * p) ** 2 + (dres / omega) ** 2 + g ** 2))


def unscaled_kkt(work, sc, x_s, y_s):
    """KKT residuals of the original problem (pdlp.py:497-520)."""
    x = sc.unscale_primal(x_s)
    y = sc.unscale_dual(y_s)
    A = work["A"]
    ax = A.matvec(x)
    pv = np.maximum(work["row_lb"] - ax, 0.0) + np.maximum(ax - work["row_ub"], 0.0)
    bv = np.maximum(work["col_lb"] - x, 0.0) + np.maximum(x - work["col_ub"], 0.0)
    primal_res = float(max(np.abs(pv).max(initial=0.0), np.abs(bv).max(initial=0.0)))
    d = work["c"] + A.rmatvec(y)
    lo_fin = work["col_lb"] > -INF
    hi_fin = work["col_ub"] < INF
    dres = np.where(lo_fin, 0.0, np.maximum(d, 0.0)) + \
        np.where(hi_fin, 0.0, np.maximum(-d, 0.0))
    dual_res = float(np.abs(dres).max(initial=0.0))
    pobj = float(work["c"] @ x) + work["obj_offset"]
    supp = np.where(y > 0.0, np.where(work["row_ub"] < INF, work["row_ub"], 0.0),
                    np.where(work["row_lb"] > -INF, work["row_lb"], 0.0)) * y
    bnd = np.where(d > 0.0, np.where(lo_fin, work["col_lb"], 0.0),
                   np.where(hi_fin, work["col_ub"], 0.0)) * d
    dobj = float(-supp.sum() + bnd.sum()) + work["obj_offset"]
    return primal_res, dual_res, abs(pobj - dobj), pobj, dobj


def converged(p, d, g, pobj, dobj, prob, params):
    """pdlp.py:523-530: feasibility capped absolutely, optimality relative."""
    rl = np.asarray(prob.row_lb, dtype=np.float64)
    ru = np.asarray(prob.row_ub, dtype=np.float64)
    c = np.asarray(prob.c, dtype=np.float64)
    rhs = max(float(np.abs(np.where(rl > -INF, rl, 0.0)).max(initial=0.0)),
              float(np.abs(np.where(ru < INF, ru, 0.0)).max(initial=0.0)))
    cn = float(np.abs(c).max(initial=0.0))
    eps_abs, eps_rel = _param(params, "eps_abs"), _param(params, "eps_rel")
    cap = _param(params, "feas_cap")
    ptol = min(eps_abs + eps_rel * rhs, cap)
    dtol = min(eps_abs + eps_rel * cn, cap)
    return (p <= ptol and d <= dtol
            and g <= eps_abs + eps_rel * (abs(pobj) + abs(dobj)))


def solve_pdlp(prob, params=None, max_seconds=None):
    """Restarted averaged PDHG, pdlp.py:238-494, on the CPU.

    ``max_seconds`` (oracle-only) stops the loop early at a check boundary
    and is used only to time a bounded sample; with it unset the loop is the
    reference's.  Returns a namespace with the fields of the reference's
    ``Solution`` plus ``info`` and ``scaling``."""
    P = (lambda name: _param(params, name))
    t0 = time.perf_counter()
    if getattr(prob, "Q", None) is not None:
        raise ValueError("oracle PDLP is for LPs (Q is None)")
    flip = int(prob.sense) == MAXIMISE
    c_work = -np.asarray(prob.c, dtype=np.float64) if flip else np.asarray(prob.c, dtype=np.float64)
    off_work = -float(prob.obj_offset) if flip else float(prob.obj_offset)
    work_prob = SimpleNamespace(A=prob.A, c=c_work, row_lb=prob.row_lb, row_ub=prob.row_ub,
                                col_lb=prob.col_lb, col_ub=prob.col_ub, obj_offset=off_work,
                                kind=getattr(prob, "kind", None))
    S, sc = scale_problem(work_prob, method=P("scaling"))
    A = S.A
    m, n = S.m, S.n
    work = dict(A=Mat.of(prob.A), c=c_work,
                row_lb=np.asarray(prob.row_lb, dtype=np.float64),
                row_ub=np.asarray(prob.row_ub, dtype=np.float64),
                col_lb=np.asarray(prob.col_lb, dtype=np.float64),
                col_ub=np.asarray(prob.col_ub, dtype=np.float64),
                obj_offset=off_work)

    c, rl, ru, lo, hi = S.c, S.row_lb, S.row_ub, S.col_lb, S.col_ub
    kkt = KKT(S)

    x = np.clip(np.zeros(n), lo, hi)
    y = np.zeros(m)
    ax = A.matvec(x)
    aty = A.rmatvec(y)

    anorm = estimate_norm(A)
    eta = 1.0 / anorm

    cn = float(np.linalg.norm(c))
    bn = float(np.linalg.norm(np.where(rl > -INF, rl, 0.0) + np.where(ru < INF, ru, 0.0)))
    omega = float(np.exp(np.log(max(cn, 1e-12)) - np.log(max(bn, 1e-12)))) if bn > 0 else 1.0
    omega = float(np.clip(omega, 1e-4, 1e4))

    sum_x = np.zeros(n)
    sum_y = np.zeros(m)
    sum_eta = 0.0
    x_restart = x.copy()
    y_restart = y.copy()
    mu_restart = kkt.merit(x, y, omega, ax, aty)
    mu_last = float("inf")
    epoch_iters = 0

    info = Info(device="cpu")
    status = ITERATION_LIMIT
    k = 0
    attempts = 0
    check_every, stepsize_every = P("check_every"), P("stepsize_every")
    max_iter, time_limit = P("max_iter"), P("time_limit")
    beta_s, beta_n, beta_a = P("beta_sufficient"), P("beta_necessary"), P("beta_artificial")
    theta = P("primal_weight_smoothing")

    while k < max_iter:
        if k % check_every == 0:
            el = time.perf_counter() - t0
            if el > time_limit:
                status = TIME_LIMIT
                break
            if max_seconds is not None and el > max_seconds:
                break
        adapt = (k % stepsize_every) == 0
        if adapt:
            accepted = False
            for _ in range(60):
                attempts += 1
                tau = eta / omega
                sigma = eta * omega
                x_new = np.clip(x - tau * (c + aty), lo, hi)   # backend.py:404-409
                dx = x_new - x
                adx = A.matvec(dx)
                ax_bar = ax + 2.0 * adx
                w = y + sigma * ax_bar                        # backend.py:417-428
                pr = np.clip(w / sigma, rl, ru)
                y_new = w - sigma * pr
                dy = y_new - y
                interaction = abs(float(np.dot(dy, adx)))
                movement = 0.5 * (omega * float(np.dot(dx, dx))
                                  + float(np.dot(dy, dy)) / omega)
                if movement == 0.0:
                    accepted = True
                    break
                eta_limit = movement / interaction if interaction > 0 else float("inf")
                t = attempts + 1
                eta_next = max(min((1.0 - t ** -0.3) * eta_limit,
                                   (1.0 + t ** -0.6) * eta), 1e-14)
                if eta <= eta_limit:
                    accepted = True
                    eta = eta_next
                    break
                info.rejected_steps += 1
                eta = eta_next
            if not accepted:
                status = NUMERICAL
                break
            ady = A.rmatvec(dy)
            x = x_new
            y = y_new
            ax += adx
            aty += ady
            sum_x += eta * x
            sum_y += eta * y
        else:
            tau = eta / omega
            sigma = eta * omega
            xnew = np.clip(x - tau * (c + aty), lo, hi)        # backend.py:441-447
            dx = xnew - x
            x[...] = xnew
            adx = A.matvec(dx)
            ax += adx                                          # backend.py:454-462
            w = y + sigma * (ax + adx)
            ynew = w - sigma * np.clip(w / sigma, rl, ru)
            dy = ynew - y
            y[...] = ynew
            ady = A.rmatvec(dy)
            aty += ady                                         # backend.py:469-474
            sum_x += eta * x
            sum_y += eta * y
        sum_eta += eta
        k += 1
        epoch_iters += 1

        if k % check_every == 0:
            p, dres, g, pobj, dobj = kkt(x, y, ax, aty)
            mu_c = float(np.sqrt((omega * p) ** 2 + (dres / omega) ** 2 + g ** 2))
            if sum_eta > 0:
                avg_x = sum_x / sum_eta
                avg_y = sum_y / sum_eta
                mu_a = kkt.merit(avg_x, avg_y, omega)
            else:
                avg_x, avg_y, mu_a = x, y, float("inf")
            use_avg = mu_a < mu_c
            mu_cand = mu_a if use_avg else mu_c
            cand_x = avg_x if use_avg else x
            cand_y = avg_y if use_avg else y
            pu, du, gu, pou, dou = unscaled_kkt(work, sc, cand_x, cand_y)
            if converged(pu, du, gu, pou, dou, prob, params):
                x, y = cand_x, cand_y
                status = OPTIMAL
                info.primal_res, info.dual_res, info.gap = pu, du, gu
                info.primal_obj, info.dual_obj = pou, dou
                break
            info.history.append((k, pu, du, gu, pou))
            do_restart = (
                mu_cand <= beta_s * mu_restart
                or (mu_cand <= beta_n * mu_restart and mu_cand > mu_last)
                or epoch_iters >= beta_a * max(k, 1)
            )
            mu_last = mu_cand
            if do_restart:
                x = cand_x.copy()
                y = cand_y.copy()
                ax = A.matvec(x)
                aty = A.rmatvec(y)
                ddx = float(np.linalg.norm(x - x_restart))
                ddy = float(np.linalg.norm(y - y_restart))
                if ddx > 1e-12 and ddy > 1e-12:
                    omega = float(np.exp(theta * np.log(ddy / ddx)
                                         + (1.0 - theta) * np.log(omega)))
                    omega = float(np.clip(omega, 1e-6, 1e6))
                x_restart, y_restart = x.copy(), y.copy()
                mu_restart = mu_cand
                sum_x = np.zeros(n)
                sum_y = np.zeros(m)
                sum_eta = 0.0
                epoch_iters = 0
                info.restarts += 1

    x_orig = sc.unscale_primal(x)
    x_orig = np.clip(x_orig, np.asarray(prob.col_lb, dtype=np.float64),
                     np.asarray(prob.col_ub, dtype=np.float64))
    y_orig = -sc.unscale_dual(y)
    obj = float(np.asarray(prob.c, dtype=np.float64) @ x_orig) + float(prob.obj_offset)
    if flip:
        y_orig = -y_orig
    info.iterations = k
    info.step_size = eta
    info.primal_weight = omega
    d = np.asarray(prob.c, dtype=np.float64) - Mat.of(prob.A).rmatvec(y_orig)
    has = status in _HAS_SOLUTION
    return SimpleNamespace(
        status=status, status_name=STATUS_NAMES[status], x=x_orig,
        objective=obj if has else float("nan"), y=y_orig, reduced_costs=d,
        iterations=k, time=time.perf_counter() - t0, method="pdlp[cpu]",
        log=info.history, dual_bound=obj if has else float("nan"),
        work_units=float(k), info=info, scaling=sc)
