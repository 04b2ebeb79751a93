"""CPU restatement of the reference's independent verifier -- TEST INFRASTRUCTURE.

``verify(prob, x, claimed_obj, feas_tol, y=..., opt_tol)`` follows
``bench/verify.py:194-276``: column bounds, row activities through the
compensated residual (``src/sovopt/numerics/refine.py:49-87,113-120``),
objective recomputation, and -- when duals are given for a continuous model --
the certified Neumaier-Shcherbina bound of ``src/sovopt/mip/safebound.py``
(``certified_bound`` 252-307, ``safe_dual_bound`` 91-133 with ``strict=True``).
It recomputes everything from the model and the point; it never looks at what
the solver computed besides ``x``, ``y`` and the claimed objective.
"""

from __future__ import annotations

import ctypes

import numpy as np

from .pdlp_oracle import INF, Mat, compensated_residual, lib

MAXIMISE = -1


def _neumaier(a):
    """safebound.py:161-171, in C (oracle/sparse_ref.c: neumaier_sum)."""
    a = np.ascontiguousarray(a, dtype=np.float64)
    L = lib()
    fn = L.neumaier_sum
    fn.argtypes = [ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    s = ctypes.c_double()
    c = ctypes.c_double()
    fn(a.shape[0], a.ctypes.data, ctypes.byref(s), ctypes.byref(c))
    return s.value, c.value


def _term(coef, lo, hi):
    """safebound.py:91-97."""
    pos = coef > 0.0
    chosen = np.where(pos, lo, hi)
    bad = np.where(pos, lo <= -INF, hi >= INF) & (coef != 0.0)
    return np.where(bad, -np.inf, coef * np.where(bad, 0.0, chosen))


def safe_dual_bound(A: Mat, c, rl, ru, lo, hi, y, strict=False, zero=None):
    """safebound.py:100-143 (textbook sign: d = c - Aᵀy)."""
    y = np.asarray(y, dtype=np.float64)
    y = np.where((y > 0.0) & (rl <= -INF), 0.0, y)
    y = np.where((y < 0.0) & (ru >= INF), 0.0, y)
    d = c - A.rmatvec(y)
    if zero is not None:
        d = np.where(zero, 0.0, d)
    row_terms = _term(y, rl, ru)
    col_terms = _term(d, lo, hi)
    if not np.isfinite(row_terms).all() or not np.isfinite(col_terms).all():
        return -np.inf
    if strict:
        total, comp = _neumaier(row_terms)
        t2, c2 = _neumaier(col_terms)
        total, comp = total + t2, comp + c2
        value = total + comp
        eps = np.finfo(np.float64).eps
        mag = float(np.abs(row_terms).sum() + np.abs(col_terms).sum())
        return float(value - 4.0 * eps * mag)
    return float(row_terms.sum() + col_terms.sum())


def certified_bound(prob, x, y, dual_tol=1e-6):
    """safebound.py:252-307 for an LP (Q is None)."""
    A = Mat.of(prob.A)
    y = np.asarray(y, dtype=np.float64)
    c = np.asarray(prob.c, dtype=np.float64)
    off = float(prob.obj_offset)
    if int(prob.sense) == MAXIMISE:
        c, off, y = -c, -off, -y
    rl = np.asarray(prob.row_lb, dtype=np.float64)
    ru = np.asarray(prob.row_ub, dtype=np.float64)
    lo = np.asarray(prob.col_lb, dtype=np.float64)
    hi = np.asarray(prob.col_ub, dtype=np.float64)
    yy = np.where((y > 0.0) & (rl <= -INF), 0.0, y)
    yy = np.where((yy < 0.0) & (ru >= INF), 0.0, yy)
    d = c - A.rmatvec(yy)
    bad = ((d > 0.0) & (lo <= -INF)) | ((d < 0.0) & (hi >= INF))
    scale = 1.0 + float(np.abs(c).max(initial=0.0))
    pert = float(np.abs(d[bad]).max(initial=0.0))
    zero = None
    if bad.any() and pert <= dual_tol * scale:
        zero = bad
    else:
        pert = 0.0 if not bad.any() else pert
    b = safe_dual_bound(A, c, rl, ru, lo, hi, yy, strict=True, zero=zero) + off
    return (-b if int(prob.sense) == MAXIMISE else b), pert


class Verdict:
    """bench/verify.py:55-113 (checks list and ``ok``)."""

    def __init__(self):
        self.checks = []
        self.certified_bound = None
        self.gap_rel = None

    def add(self, name, ok, detail=""):
        self.checks.append((name, bool(ok), detail))

    @property
    def ok(self):
        return all(c[1] for c in self.checks)

    def failed(self):
        return [c for c in self.checks if not c[1]]

    def report(self):
        return "\n".join(f"  [{'PASS' if ok else 'FAIL'}] {n}  {d}" for n, ok, d in self.checks)


def verify(prob, x, claimed_obj=None, feas_tol=1e-6, int_tol=1e-6, y=None, opt_tol=1e-9):
    """bench/verify.py:194-276."""
    v = Verdict()
    x = np.asarray(x, dtype=np.float64)
    A = Mat.of(prob.A)
    if x.shape[0] != A.n:
        v.add("dimension", False, f"got {x.shape[0]}, model has {A.n} columns")
        return v
    v.add("dimension", True, f"{A.n} columns")
    if not np.isfinite(x).all():
        v.add("finite", False, "solution contains NaN or Inf")
        return v
    v.add("finite", True, "")
    lo = np.asarray(prob.col_lb, dtype=np.float64)
    hi = np.asarray(prob.col_ub, dtype=np.float64)
    rl = np.asarray(prob.row_lb, dtype=np.float64)
    ru = np.asarray(prob.row_ub, dtype=np.float64)
    lo_v = float(np.maximum(lo - x, 0.0).max(initial=0.0))
    hi_v = float(np.maximum(x - hi, 0.0).max(initial=0.0))
    bnd = max(lo_v, hi_v)
    v.add("column bounds", bnd <= feas_tol, f"max violation {bnd:.3e}")
    act = -compensated_residual(A.rp, A.ri, A.rx, x, np.zeros(A.m))
    rlo = float(np.maximum(rl - act, 0.0).max(initial=0.0))
    rhi = float(np.maximum(act - ru, 0.0).max(initial=0.0))
    rowv = max(rlo, rhi)
    v.add("row constraints", rowv <= feas_tol, f"max violation {rowv:.3e}")
    kind = getattr(prob, "kind", None)
    mask = (np.asarray(kind) == 1) | (np.asarray(kind) == 2) if kind is not None \
        else np.zeros(A.n, dtype=bool)
    if mask.any():
        iv = float(np.abs(x[mask] - np.round(x[mask])).max(initial=0.0))
        v.add("integrality", iv <= int_tol, f"max distance to integer {iv:.3e}")
    else:
        v.add("integrality", True, "no integer variables")
    obj = float(np.asarray(prob.c, dtype=np.float64) @ x) + float(prob.obj_offset)
    if claimed_obj is not None:
        d = abs(obj - claimed_obj) / max(1.0, abs(obj))
        v.add("objective", d <= 1e-6,
              f"recomputed {obj:.12g}, claimed {claimed_obj:.12g}, rel diff {d:.2e}")
    else:
        v.add("objective", True, f"recomputed {obj:.12g}")
    if y is not None and not mask.any():
        y = np.asarray(y, dtype=np.float64)
        if y.shape[0] != A.m or not np.isfinite(y).all():
            v.add("optimality", False, "dual vector has the wrong length or is not finite")
        else:
            bound, pert = certified_bound(prob, x, y)
            v.certified_bound = bound
            if not np.isfinite(bound):
                v.gap_rel = float("inf")
                v.add("optimality", False, f"the duals certify nothing ({pert:.2e})")
            else:
                gap = (obj - bound) if int(prob.sense) != MAXIMISE else (bound - obj)
                rel = gap / max(1.0, abs(obj))
                v.gap_rel = rel
                if rel < -opt_tol:
                    v.add("optimality", False, f"objective {gap:.3e} below the certified bound")
                else:
                    v.add("optimality", rel <= opt_tol,
                          f"certified bound {bound:.12g}, gap {gap:.3e} ({rel:.2e} relative)")
    return v


def verify_files(prob, solution_path, feas_tol=1e-6, int_tol=1e-6):
    """bench/verify.py:279-318 without the MPS read: the solution file is a
    JSON payload with ``x`` (list or name-keyed object), optional ``objective``
    and optional ``y`` (list or name-keyed object), or a bare list of x."""
    import json
    with open(solution_path, encoding="utf-8") as fh:
        data = json.load(fh)
    y = None
    if isinstance(data, dict) and "x" in data:
        if isinstance(data["x"], dict):
            names = {nm: i for i, nm in enumerate(prob.col_names or [])}
            x = np.zeros(prob.A.n)
            for nm, val in data["x"].items():
                if nm in names:
                    x[names[nm]] = val
        else:
            x = np.asarray(data["x"], dtype=float)
        claimed = data.get("objective")
        if data.get("y") is not None:
            if isinstance(data["y"], dict):
                rnames = {nm: i for i, nm in enumerate(prob.row_names or [])}
                y = np.zeros(prob.A.m)
                for nm, val in data["y"].items():
                    if nm in rnames:
                        y[rnames[nm]] = val
            else:
                y = np.asarray(data["y"], dtype=float)
    else:
        x = np.asarray(data, dtype=float)
        claimed = None
    return verify(prob, x, claimed, feas_tol, int_tol, y=y)
