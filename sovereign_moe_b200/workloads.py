"""Seeded synthetic LPs with a known optimum.

Every generator builds ``min cᵀx  s.t.  Ax = b,  0 <= x <= u`` so that the
optimum is known exactly by construction:

* ``u ~ U(1, 10)``; ``x*`` has 30% of its entries at 0, 30% at ``u`` and the
  rest at ``U(0.1, 0.9)·u``;
* ``y* ~ N(0, 1)``, ``b = A x*``;
* ``z`` with ``|z| ~ U(0.1, 1)``, ``z >= 0`` where ``x* = 0``, ``z <= 0`` where
  ``x* = u`` and 0 elsewhere; ``c = Aᵀy* + z``.

Then ``c - Aᵀy* = z`` has the sign complementarity demands at ``x*``, so
``(x*, y*)`` is a KKT pair and ``f* = cᵀx*`` is the optimal value.  Rows are
equalities (``rl = ru = b``), columns are boxed.

The five workloads (sizes as the benchmark configuration states them):

* :func:`single_small`   -- 230 x 2,025, exactly 6 nnz per column, N(0,1);
* :func:`blending_plan`  -- 200,000 x 600,000, 5 nnz per column (3M), a
  720-period blending plan: intra-period rows, block-bidiagonal inventory links
  to period t+1, 30 global coupling rows, values log-uniform in ±[1e-3, 1e3];
* :func:`uneven_batch`   -- 256 LPs, rows log-uniform in [50, 5000], columns
  U{2..8}·rows, 4-12 nnz per column, N(0,1);
* :func:`power_law`      -- 1M x 3M, 10M nnz, Zipf(1.5) column degrees capped at
  2,000 and rescaled to the total, N(0,1) with 1% of rows scaled by 1e4;
* :func:`serving_stream` -- Poisson arrivals of LPs from a size mixture (70%
  100-2k rows, 25% 2k-50k, 5% 50k-300k), U{2..8}·rows columns, 3-10 nnz per
  column.

Public benchmark sets are not available offline; these seeded constructions
stand in for them, with the shapes, sizes and value distributions above.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .problem import Problem, SparseMatrix

__all__ = ["KnownLP", "known_optimum", "single_small", "blending_plan",
           "uneven_batch", "power_law", "serving_stream", "random_structure"]


@dataclass
class KnownLP:
    """A generated LP and the optimum it was built around."""
    problem: Problem
    f_star: float
    x_star: np.ndarray
    y_star: np.ndarray


def _fix_duplicates(rng, col, rows, lo, span, max_rounds=200):
    """Redraw entries until no column holds a row twice.  ``lo``/``span`` give,
    per entry, the half-open row range the entry is drawn from."""
    m_key = np.int64(max(int((lo + span).max(initial=1)), 1))
    for _ in range(max_rounds):
        key = col.astype(np.int64) * m_key + rows
        order = np.argsort(key, kind="stable")
        ks = key[order]
        dup = np.zeros(ks.shape[0], dtype=bool)
        if ks.shape[0] > 1:
            dup[1:] = ks[1:] == ks[:-1]
        if not dup.any():
            return rows
        pos = order[dup]
        rows[pos] = lo[pos] + rng.integers(0, span[pos])
    raise RuntimeError("could not draw distinct rows; a column degree is too close to its row range")


def random_structure(rng, m, degrees, lo=None, span=None):
    """CSC pattern with ``degrees[j]`` distinct rows in column ``j``, drawn
    uniformly from ``[lo, lo + span)`` per entry (default: all rows)."""
    degrees = np.asarray(degrees, dtype=np.int64)
    n = degrees.shape[0]
    cp = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(degrees, out=cp[1:])
    nnz = int(cp[-1])
    col = np.repeat(np.arange(n, dtype=np.int64), degrees)
    if lo is None:
        lo = np.zeros(nnz, dtype=np.int64)
        span = np.full(nnz, m, dtype=np.int64)
    rows = lo + rng.integers(0, span)
    rows = _fix_duplicates(rng, col, rows, lo, span)
    order = np.lexsort((rows, col))
    return cp, rows[order].astype(np.int32)


def known_optimum(rng, m, n, cp, ci, cx, name="known"):
    """Wrap a CSC matrix in the known-optimum construction."""
    A = SparseMatrix(m, n, cp, ci, cx)
    u = rng.uniform(1.0, 10.0, n)
    r = rng.random(n)
    at0 = r < 0.3
    atu = (r >= 0.3) & (r < 0.6)
    x_star = rng.uniform(0.1, 0.9, n) * u
    x_star[at0] = 0.0
    x_star[atu] = u[atu]
    y_star = rng.standard_normal(m)
    b = A.matvec(x_star)
    mag = rng.uniform(0.1, 1.0, n)
    z = np.zeros(n)
    z[at0] = mag[at0]
    z[atu] = -mag[atu]
    c = A.rmatvec(y_star) + z
    prob = Problem(A=A, c=c, row_lb=b.copy(), row_ub=b.copy(),
                   col_lb=np.zeros(n), col_ub=u, name=name)
    return KnownLP(prob, float(c @ x_star), x_star, y_star)


def single_small(seed=0, m=230, n=2025, per_col=6):
    """230 x 2,025, exactly 6 nnz per column at uniform random rows, N(0,1)."""
    rng = np.random.default_rng(seed)
    cp, ci = random_structure(rng, m, np.full(n, per_col))
    cx = rng.standard_normal(ci.shape[0])
    return known_optimum(rng, m, n, cp, ci, cx, name=f"small_{m}x{n}_s{seed}")


def _log_uniform_signed(rng, size, lo=1e-3, hi=1e3):
    mag = np.exp(rng.uniform(np.log(lo), np.log(hi), size))
    return np.where(rng.random(size) < 0.5, -mag, mag)


def blending_plan(seed=0, m=200_000, n=600_000, per_col=5, periods=720,
                  coupling=30, link_frac=0.10, couple_frac=0.05):
    """A multi-period blending plan: each period owns a band of rows and
    columns; ``link_frac`` of a period's columns also enter a row of the next
    period (the inventory link, making the matrix block-bidiagonal), and
    ``couple_frac`` enter one of the ``coupling`` global capacity rows."""
    rng = np.random.default_rng(seed)
    prow = m - coupling
    r_edges = np.linspace(0, prow, periods + 1).round().astype(np.int64)
    c_edges = np.linspace(0, n, periods + 1).round().astype(np.int64)
    period_of_col = np.searchsorted(c_edges, np.arange(n), side="right") - 1
    degrees = np.full(n, per_col, dtype=np.int64)
    nnz = n * per_col
    col = np.repeat(np.arange(n, dtype=np.int64), degrees)
    slot = np.tile(np.arange(per_col, dtype=np.int64), n)
    t = period_of_col[col]
    lo = r_edges[t].copy()
    span = (r_edges[t + 1] - r_edges[t]).copy()
    is_link = rng.random(n) < link_frac
    is_link &= period_of_col < periods - 1
    is_couple = rng.random(n) < couple_frac
    link_e = is_link[col] & (slot == per_col - 1)
    lo[link_e] = r_edges[t[link_e] + 1]
    span[link_e] = r_edges[t[link_e] + 2] - r_edges[t[link_e] + 1]
    couple_e = is_couple[col] & (slot == per_col - 2)
    lo[couple_e] = prow
    span[couple_e] = coupling
    rows = lo + rng.integers(0, span)
    rows = _fix_duplicates(rng, col, rows, lo, span)
    order = np.lexsort((rows, col))
    cp = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(degrees, out=cp[1:])
    ci = rows[order].astype(np.int32)
    cx = _log_uniform_signed(rng, nnz)
    return known_optimum(rng, m, n, cp, ci, cx, name=f"blend_{m}x{n}_s{seed}")


def uneven_batch(seed=0, count=256, m_lo=50, m_hi=5000):
    """``count`` LPs: rows log-uniform in [m_lo, m_hi], columns U{2..8}·rows,
    4-12 nnz per column (capped at the row count), N(0,1)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        m = int(round(np.exp(rng.uniform(np.log(m_lo), np.log(m_hi)))))
        n = int(rng.integers(2, 9)) * m
        sub = np.random.default_rng([seed, i])
        deg = np.minimum(sub.integers(4, 13, n), m)
        cp, ci = random_structure(sub, m, deg)
        cx = sub.standard_normal(ci.shape[0])
        out.append(known_optimum(sub, m, n, cp, ci, cx, name=f"batch{i}_{m}x{n}"))
    return out


def node_relaxation(seed=1234, m=20_000, n=30_000, per_col=8, nodes=128):
    """A 20,000 x 30,000 LP with 8 nnz per column (uniform random rows,
    N(0,1) values) around an interior point x0 ~ U[0,1): rows A x = A x0,
    costs N(0,1), columns in [0, 10] -- the matrix shape the reference
    benchmarks batched node relaxation on (bench/gpu_bench.py:31-44, 173).
    There the rows are A x <= A x0 + U[0, 0.5); here they are equalities,
    because the reference's safe dual bound (safebound.py:212-230) prices a
    positive dual at the row's lower bound and a negative one at its upper
    bound, while its PDHG step (bnr.py:238-242) gives a one-sided row the
    dual sign whose price is infinite, so every bound of that LP would be
    -inf.  Also ``nodes`` branch-and-bound-like bound sets (n, nodes): node k
    halves the box of 3 random columns.  Returns (problem, L, U)."""
    rng = np.random.default_rng(seed)
    cp, ci = random_structure(rng, m, np.full(n, per_col))
    cx = rng.standard_normal(ci.shape[0])
    A = SparseMatrix(m, n, cp, ci, cx)
    x0 = rng.random(n)
    b = A.matvec(x0)
    prob = Problem(A=A, c=rng.standard_normal(n), row_lb=b, row_ub=b.copy(),
                   col_lb=np.zeros(n), col_ub=np.full(n, 10.0), name=f"nodes_{m}x{n}")
    L = np.zeros((n, nodes))
    U = np.full((n, nodes), 10.0)
    for k in range(nodes):
        j = rng.choice(n, size=3, replace=False)
        lower = rng.random(3) < 0.5
        U[j[lower], k] = 5.0
        L[j[~lower], k] = 5.0
    return prob, L, U


def power_law(seed=0, m=1_000_000, n=3_000_000, nnz=10_000_000, alpha=1.5,
              cap=2000, heavy_rows=0.01, heavy_scale=1e4):
    """Zipf(alpha) column degrees capped at ``cap`` and rescaled so they sum to
    ``nnz``; N(0,1) values with ``heavy_rows`` of the rows scaled by
    ``heavy_scale``."""
    rng = np.random.default_rng(seed)
    d = np.minimum(rng.zipf(alpha, n), cap).astype(np.float64)
    d *= nnz / d.sum()
    base = np.floor(d)
    deg = (base + (rng.random(n) < (d - base))).astype(np.int64)
    deg = np.clip(deg, 1, min(cap, m))
    diff = int(nnz - deg.sum())
    while diff != 0:
        j = rng.integers(0, n, abs(diff))
        if diff > 0:
            j = j[deg[j] < min(cap, m)]
            np.add.at(deg, j, 1)
        else:
            j = j[deg[j] > 1]
            np.add.at(deg, j, -1)
        deg = np.clip(deg, 1, min(cap, m))
        diff = int(nnz - deg.sum())
    cp, ci = random_structure(rng, m, deg)
    cx = rng.standard_normal(ci.shape[0])
    heavy = rng.random(m) < heavy_rows
    cx = np.where(heavy[ci], cx * heavy_scale, cx)
    return known_optimum(rng, m, n, cp, ci, cx, name=f"powerlaw_{m}x{n}_s{seed}")


def serving_stream(seed=0, count=64, rate=100.0, classes=((0.70, 100, 2000),
                   (0.25, 2000, 50_000), (0.05, 50_000, 300_000)), max_rows=None):
    """``count`` LPs with Poisson arrival times at ``rate`` per second.  Row
    counts come from the size mixture (log-uniform within a class), columns
    are U{2..8}·rows, 3-10 nnz per column.  ``max_rows`` caps the draw (for
    tests).  Returns ``[(arrival_seconds, KnownLP), ...]``."""
    rng = np.random.default_rng(seed)
    probs = np.array([c[0] for c in classes])
    t = np.cumsum(rng.exponential(1.0 / rate, count))
    out = []
    for i in range(count):
        k = int(rng.choice(len(classes), p=probs / probs.sum()))
        _, lo, hi = classes[k]
        m = int(round(np.exp(rng.uniform(np.log(lo), np.log(hi)))))
        if max_rows is not None:
            m = min(m, max_rows)
        n = int(rng.integers(2, 9)) * m
        sub = np.random.default_rng([seed, i, 7])
        deg = np.minimum(sub.integers(3, 11, n), m)
        cp, ci = random_structure(sub, m, deg)
        cx = sub.standard_normal(ci.shape[0])
        out.append((float(t[i]), known_optimum(sub, m, n, cp, ci, cx,
                                               name=f"serve{i}_{m}x{n}")))
    return out
